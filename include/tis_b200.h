/*
 * tis_b200.h -- C-ABI of the B200 (sm_100a) force-and-integrate library for
 * the TIS coarse-grained RNA engine (DT15 model).
 *
 * Every array crossing this boundary is caller-owned HOST memory laid out the
 * way the Fortran host keeps it (column-major, xyz fastest), indices inside
 * topology arrays are 1-based bead numbers, and replica arguments are 1-based
 * (`irep`), exactly as the Fortran module globals of the reference:
 *
 *   xyz_mp_rep(3, nmp_all, nrep), velo_mp(3, nmp_real, nrep),
 *   accel_mp(3, nmp_real, nrep), force_mp(3, nmp_all), energy(E_TYPE%MAX)
 *   (src/var_struct.F90, src/var_simu.F90 of the reference).
 *
 * Return codes: 0 ok, >0 warning count (force clamps at DE_MAX), <0 fatal
 * (see TIS_E_* below).  The library never calls exit().  One context per
 * host thread; calls on one context are not reentrant.
 */
#ifndef TIS_B200_H
#define TIS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ enums */
/* Values of the reference's enums (src/const_index.F90:88-97, 99-145, 225-241). */
enum {
  TIS_CLASS_RNA = 2,
  TIS_CLASS_LIG = 3,
  TIS_CLASS_ION = 4
};
enum {
  TIS_MP_RNA_PHOS = 2,
  TIS_MP_RNA_BASE = 3,
  TIS_MP_RNA_SUGAR = 4,
  TIS_MP_ION_MG = 5,
  TIS_MP_ION_CA2 = 6,
  TIS_MP_ION_NA = 7,
  TIS_MP_ION_K = 8,
  TIS_MP_ION_CL = 9
};
/* E_TYPE (1-based in Fortran; index E-1 in C arrays of length TIS_ETYPE_MAX). */
enum {
  TIS_E_TOTAL = 1, TIS_E_VELO = 2, TIS_E_BOND = 3, TIS_E_BANGLE = 4,
  TIS_E_ELE = 8, TIS_E_STACK_DTRNA = 16, TIS_E_HBOND_DTRNA = 17,
  TIS_E_EXV_DT15 = 18, TIS_E_TSTACK_DTRNA = 19, TIS_E_THBOND_DTRNA = 20,
  TIS_E_WCA_REP = 23, TIS_E_WCA_ATT = 24,
  TIS_ETYPE_MAX = 25
};
/* i_hydro_tensor values (src/const_index.F90:39-45 HI_TENSOR). */
enum { TIS_HI_RPY = 1, TIS_HI_RPY_OVER = 2, TIS_HI_ERMAK_OVER = 3, TIS_HI_ZUK_RPY = 4 };
/* i_simulate_type values used here (src/const_index.F90 SIM). */
enum { TIS_SIM_LANGEVIN = 1, TIS_SIM_BROWNIAN_HI = 6 };
/* electrostatics: 0 none, DH = i_function_form 0, EWALD = i_function_form 2,
 * COULOMB = i_function_form 1 (plain Coulomb with a cutoff in A,
 * src/force_ele_coulomb.F90, src/energy_ele_coulomb.F90) */
enum { TIS_ELE_NONE = 0, TIS_ELE_DH = 1, TIS_ELE_EWALD = 2, TIS_ELE_COULOMB = 3 };
/* arithmetic of the force terms */
enum { TIS_PREC_FP64 = 0, TIS_PREC_MIXED = 1 };

/* error codes */
#define TIS_OK 0
#define TIS_E_ARG (-1)
#define TIS_E_CUDA (-2)
#define TIS_E_LIST_OVERFLOW (-3)
#define TIS_E_NOT_SPD (-4)
#define TIS_E_TIMEOUT (-5)
#define TIS_E_NOISE_EXHAUSTED (-6)
#define TIS_E_UNSUPPORTED (-7)
#define TIS_E_NAN (-8)
#define TIS_E_PMF_RANGE (-9)   /* a Mg-P pair came closer than the PMF table's first point (the reference stops: force_ele_DH.F90:90-93) */

/* -------------------------------------------------------------- topology */
/* One system (unit list + DT15 interaction tables) as read_nativeinfo and
 * setp_dtrna15 leave it (src/read_nativeinfo.F90:121-620,833-986,
 * src/setp_dtrna15.F90:40-174).  All index arrays hold 1-based bead numbers. */
typedef struct tis_topology {
  int32_t nmp;                     /* nmp_all (= nmp_real: no virtual beads) */
  int32_t nunit;
  const int32_t *lunit2mp;         /* (2, nunit) first/last bead of each unit */
  const int32_t *iclass_unit;      /* (nunit) TIS_CLASS_* */
  const int32_t *imp2type;         /* (nmp) TIS_MP_* */
  const double *cmass;             /* (nmp) cmass_mp */
  const double *fric;              /* (nmp) fric_mp (mass-divided for Langevin) */
  const double *exv_radius;        /* (nmp) exv_radius_mp */
  const double *exv_epsilon;       /* (nmp) exv_epsilon_mp = sqrt(eps) */
  int32_t ncharge;
  const int32_t *icharge2mp;       /* (ncharge), increasing */
  const double *coef_charge;       /* (ncharge) */
  int32_t nbd;                     /* harmonic bonds */
  const int32_t *ibd2mp;           /* (2, nbd) */
  const double *bd_nat;            /* (nbd) */
  const double *coef_bd;           /* (nbd) */
  int32_t nba;                     /* harmonic angles */
  const int32_t *iba2mp;           /* (3, nba) */
  const double *ba_nat;            /* (nba) radians */
  const double *coef_ba;           /* (nba) */
  int32_t nst;                     /* DT consecutive stacks */
  const int32_t *idtrna_st2mp;     /* (7, nst) B1 B2 P1 S1 P2 S2 P3 */
  const double *dtrna_st_nat;      /* (3, nst) dist, dih1, dih2 (rad) */
  const double *coef_dtrna_st;     /* (3, nst) coef 1..3 */
  const double *dtrna_st_hsTm;     /* (3, nst) h, s, Tm for U0(T) */
  int32_t nhb;                     /* DT15 hydrogen bonds */
  const int32_t *idtrna_hb2mp;     /* (6, nhb) */
  const double *dtrna_hb_nat;      /* (6, nhb) dist, 2 angles, 3 dihedrals (rad) */
  const double *coef_dtrna_hb;     /* (7, nhb) index 0 = U0, 1..6 */
  const int32_t *idtrna_hb2hbsite; /* (3, 2, nhb) 0 = unused slot */
  int32_t nhbsite;
  const int32_t *nvalence_hbsite;  /* (nhbsite) */
  int32_t nfene;                   /* FENE bonds (Brownian-HI chains) */
  const int32_t *ifene2mp;         /* (2, nfene) */
  const double *fene_nat;          /* (nfene) */
  const double *coef_fene;         /* (nfene) */
  const double *dist2_fene;        /* (nfene) */
  int32_t nwca;                    /* WCA pairs (Brownian-HI chains) */
  const int32_t *iwca2mp;          /* (2, nwca) */
  const double *wca_nat;           /* (nwca) sigma */
  const double *coef_wca;          /* (nwca, 2): repulsive, attractive */
  int32_t ntst;                    /* DT15 tertiary stacks (tbs-dist/-angl/-dihd records,
                                      src/read_nativeinfo.F90:624-700, force_dtrna_stack_nlocal.F90) */
  const int32_t *idtrna_tst2mp;    /* (6, ntst) B1 B2 S1 S2 P1' P2' */
  const double *dtrna_tst_nat;     /* (6, ntst) dist, 2 angles, 3 dihedrals (rad) */
  const double *coef_dtrna_tst;    /* (7, ntst) index 0 = U0, 1..6 */
  const int32_t *idtrna_tst2side;  /* (2, ntst) 1: the secondary stack of B with B - 3, 2: with B + 3 */
  const int32_t *flg_tst_exclusive;/* (2, ntst) nonzero: within 10 A of native, disables that stack */
  const int32_t *flg_hb_tertiary;  /* (nhb) nonzero: hb-dist record typed 'T' (src/read_nativeinfo.F90:
                                      606-613); its energy goes to TIS_E_THBOND_DTRNA instead of
                                      TIS_E_HBOND_DTRNA (energy_dtrna_hbond15.F90:135-143).  NULL:
                                      every hydrogen bond is secondary ('S') */
  const int32_t *flg_charge_fixed; /* (ncharge) nonzero: a CHARGE_CHANGE value, kept when i_charge = 1
                                      (simu_ele_set.F90:152-158).  NULL: none fixed */
  const double *radius;            /* (nmp) Brownian-HI: hydrodynamic radius of each bead (var_struct radius,
                                      setp_mass_fric.F90:91).  NULL: tis_params.hi_radius for every bead */
} tis_topology;

/* ---------------------------------------------------------------- params */
/* The inputs the reference reads from the .inp and para/ files for this
 * path (src/var_setp.F90 inperi/insimu/inele/indtrna, para/rna.para:325-416,
 * para/general.para). */
typedef struct tis_params {
  int32_t i_periodic;              /* 0 or 1 */
  double psize[3];                 /* periodic box (cubic for Ewald) */
  double neigh_margin;             /* Verlet skin, 8.0 */
  int32_t n_step_neighbor;         /* 0: skin rule (i_neigh_dynamic=1); k>0: rebuild when mod(istep,k)==1 */
  double exv_dist, exv_dist_PS, exv_adjust, exv_inf;
  int32_t n_sep_nlocal_P, n_sep_nlocal_S, n_sep_nlocal_B;
  double hb_cutoff_dist;
  int32_t i_ele;                   /* TIS_ELE_* */
  int32_t i_diele;                 /* 0 constant (diele_water), 1 Malmberg-Maryott */
  double diele_water;
  double ionic_strength;           /* mol/L */
  double cutoff_ele;               /* DH: in Debye lengths; Ewald: Angstrom */
  int32_t i_DH_cutoff_type;        /* energy only; the force always scales */
  double ewld_alpha, ewld_hmax;
  int32_t i_simulate_type;         /* TIS_SIM_* */
  double tstep;
  double viscosity;                /* Brownian-HI, internal units */
  double wca_coef_cutoff;          /* Brownian-HI WCA cutoff factor */
  int32_t precision;               /* TIS_PREC_* */
  int32_t hb_beta_global;          /* 1: reference quirk (one beta_hbond15 for all replicas) */
  uint64_t seed;                   /* counter-based noise key */
  double hi_radius;                /* Brownian-HI: Rotne-Prager bead radius (radius(1) of HI_TENSOR%RPY) */
  int32_t n_step_hydro;            /* Brownian-HI: refactor D and its Cholesky factor every n steps (reference: 1) */
  /* DT19 semi-explicit ions (i_dtrna_model = 2019) and Manning phosphate charges */
  int32_t i_dtrna_model;           /* 2015 (or 0) or 2019: base-base exv contact exv_dist, others the radius sum
                                      (force_exv_dt15.F90:60-66); no exv between a charged phosphate and an ion
                                      (neighbor_assign.F90:524-537); Mg-P pairs on the PMF + DH table */
  int32_t i_charge;                /* 0: topology charges; 1: every phosphate charge not fixed by
                                      flg_charge_fixed is -Zp of its temperature (simu_ele_set.F90:107-166) */
  double length_per_unit_P;        /* b, LENGTH_PER_UNIT of P (para/electrostatic.para: 4.38178046) */
  int32_t pmf_nbin;                /* Mg-P potential of mean force on a uniform grid (setp_pmf.F90:31-105): */
  double pmf_rmin, pmf_rbin, pmf_rmax; /* first point, spacing, last point read */
  double pmf_rmerge;               /* pmf_merge: the switch from PMF to DH (simu_ele_set.F90:242-250) */
  const double *pmf_mg_p;          /* (pmf_nbin) PMF values; NULL when the system has no Mg */
  int32_t hi_refine;               /* Brownian-HI, mixed precision: 1 refines the correlated noise once per step.
                                      The step's factor L (split-TF32 tensor-core factorisation, kept in FP32)
                                      has L L^T = D + E, |E| ~ 1e-7 |D|; the sample L xi - E L^-T xi / 2 has
                                      covariance D + O(E^2).  E is formed in FP64 at each refresh. 0: off */
  int32_t i_hydro_tensor;          /* Brownian-HI diffusion tensor (HI_TENSOR, const_index.F90:39-45): 1 (or 0)
                                      RPY, 2 RPY_OVER, 3 ERMAK_OVER (radius of bead 1), 4 ZUK_RPY (per-bead
                                      radii), simu_hydro_tensors.F90:50-324 */
  /* Launch configuration of the step kernel (no reference counterpart).  Each
   * field left 0 comes from the environment (TIS_THREADS, TIS_GROUP,
   * TIS_CLUSTER, TIS_NOISE_SWEEP), else from the measured table the
   * autotuner writes (launch_table, or tuned_launch.tsv next to the
   * library), else from a built-in rule.  The results do not depend on it
   * beyond the summation order of each bead's force. */
  int32_t launch_threads;          /* threads per CTA: 128, 256, 512, or 1024 (mixed, one CTA per replica) */
  int32_t launch_group;            /* threads per bead in the force gather: 1, 2, 4 or 8 */
  int32_t launch_ctas;             /* CTAs per replica: 1, or 2 (a cluster: mixed precision, 512 threads,
                                      no periodic box, no Ewald, >= 64 beads) */
  int32_t launch_noise_sweep;      /* two CTAs: 1 draws the noise in the bonded sweep, 2 in the update */
  int32_t launch_order;            /* 1: replicas launched in context order, 2: largest first */
  const char *launch_table;        /* NULL: tuned_launch.tsv next to the library */
  int32_t launch_sweep;            /* bonded sweep of one CTA per replica: 1 item chunks dealt to the warps
                                      in turn, 2 warps take chunks from a shared counter, longest kinds
                                      first, 3 a longest-first deal made once per launch (two CTAs: 1) */
} tis_params;

/* ---------------------------------------------------------------- status */
typedef struct tis_status_t {
  int64_t step;                    /* istep of replica 1 */
  int64_t n_rebuild;               /* neighbour rebuilds since init (all replicas) */
  int64_t n_clamp;                 /* DE_MAX clamps since last tis_status */
  int32_t list_overflow;           /* any list capacity exceeded */
  int32_t nan_seen;                /* non-finite force or coordinate seen */
  int32_t wait_timeout;            /* a bounded device wait gave up */
  int32_t not_spd;                 /* Brownian-HI Cholesky pivot <= 0 */
  int32_t last_error;              /* last TIS_E_* returned */
  int32_t exv_pairs_max;           /* largest exv half list among replicas */
  int32_t ele_pairs_max;           /* largest ele half list among replicas */
  int32_t ctas_per_lane;           /* CTAs (one cluster) that tis_step gives each replica: 1 or 2 */
  int32_t threads_per_cta;         /* the launch configuration in use (see tis_params.launch_*) */
  int32_t group;                   /* threads per bead in the force gather, 0: per-replica rule */
  int32_t noise_sweep;
  int32_t lane_order;
  int32_t launch_source;           /* 0 built-in rule, 1 tuned table, 2 caller or environment */
  int32_t sweep;
} tis_status_t;

typedef struct tis_ctx tis_ctx;

/* Builds the device context for one topology and nrep replicas whose
 * temperatures are tempk[0..nrep-1].  Replaces the allocate_xxx / setp_xxx
 * and per-stage preparation calls before mloop_simulator
 * (src/main.F90:44-58, src/main_loop.F90:89-109, src/mloop_dtrna.F90:149-155,
 * src/mloop_neigh_dist.F90:28-149, src/simu_ele_set.F90, src/simu_set_dtrna.F90). */
int tis_init(const tis_topology *top, const tis_params *par, int32_t nrep,
             const double *tempk, tis_ctx **out);

/* Uneven batch: ntop independent systems, system k replicated nrep[k] times
 * with temperatures tempk[sum(nrep[0..k-1]) ...].  No reference counterpart
 * beyond running the systems as separate processes (MXUNIT = 20). */
int tis_init_batch(int32_t ntop, const tis_topology *tops, const tis_params *par,
                   const int32_t *nrep, const double *tempk, tis_ctx **out);

/* One rank's share of a replica-exchange ladder split over processes (one
 * per GPU), as the reference distributes replicas over MPI ranks
 * (n_replica_mpi local replicas, irep2grep, var_replica.F90): the context
 * holds global replicas irep_first .. irep_first + nrep_local - 1 of an
 * nrep_all-replica ladder with temperatures tempk_all[0 .. nrep_all-1];
 * replica g starts at label g.  Counter-based noise is keyed by the global
 * replica, so a replica moves exactly as it would in one context holding the
 * whole ladder.  Exchanges go through tis_rex_energies and
 * tis_rex_exchange_all; every rank passes the same seed. */
int tis_init_ladder(const tis_topology *top, const tis_params *par, int32_t nrep_all, const double *tempk_all,
                    int32_t irep_first, int32_t nrep_local, tis_ctx **out);

void tis_destroy(tis_ctx *ctx);

/* Number of replicas (lanes) and beads of lane irep (1-based). */
int tis_nrep(const tis_ctx *ctx);
int tis_nmp(const tis_ctx *ctx, int32_t irep);

/* Copy state in / out.  xyz is xyz_mp_rep(3, nmp, nrep); pxyz_mp_rep is set
 * equal to xyz (src/simu_initial.F90); velo/accel may be NULL (zeros in,
 * skipped out).  For a batch the replicas are concatenated in lane order. */
int tis_set_state(tis_ctx *ctx, const double *xyz, const double *velo, const double *accel);
int tis_get_state(tis_ctx *ctx, double *xyz, double *velo, double *accel);
/* Periodic (wrapped) coordinates pxyz_mp_rep. */
int tis_get_pxyz(tis_ctx *ctx, double *pxyz);
/* Step counter istep of every replica (var_simu istep; read back by the
 * restart reader src/read_rst.F90 STEP block): counter-based noise and the
 * rebuild cadence continue from it. */
int tis_set_step(tis_ctx *ctx, int64_t istep);
/* DT15 hbond and stack status of replica irep (var_simu hb_status,
 * st_status as the restart's DTRNA15 block holds them, src/write_rst.F90:
 * 104-113): hb_status[ihb] = 1 when hbond ihb was on in the last force
 * evaluation (in the list, within the cutoff, not pruned); st_status[ist] =
 * 0 when a tertiary stack excludes stack ist at the current coordinates.
 * Either pointer may be NULL. */
int tis_get_dtrna_status(tis_ctx *ctx, int32_t irep, int32_t *hb_status, int32_t *st_status);

/* Parity injection.  noise: r_boxmuller(3, nmp, nrep) for nsteps consecutive
 * steps (step-major); uniforms: for each replica a stream of n_uniform draws
 * consumed in order by the hydrogen-bond valence pruning
 * (src/force_dtrna_hbond15.F90:390-509).  Pass noise == NULL / uniforms ==
 * NULL to return to the counter-based generator. */
int tis_set_noise(tis_ctx *ctx, const double *noise, int32_t nsteps,
                  const double *uniforms, int32_t n_uniform);

/* neighbor(irep): exv, ele and hbond lists (src/neighbor.F90:13-142).
 * irep = -1 rebuilds every replica. */
int tis_neighbor(tis_ctx *ctx, int32_t irep);

/* Read the lists back in the reference's layout and order:
 * iexv2mp(3, nexv) = (i, j, imirror), iele2mp(4, nele) = (i, j, imirror, ipmf)
 * with coef_ele(nele), ineigh2hb(nhbneigh).  *n receives the count; returns
 * TIS_E_LIST_OVERFLOW when cap is too small (n still set). */
int tis_get_exv_list(tis_ctx *ctx, int32_t irep, int32_t *iexv2mp, int32_t cap, int32_t *n);
int tis_get_ele_list(tis_ctx *ctx, int32_t irep, int32_t *iele2mp, double *coef_ele,
                     int32_t cap, int32_t *n);
int tis_get_hb_list(tis_ctx *ctx, int32_t irep, int32_t *ineigh2hb, int32_t cap, int32_t *n);

/* force_sumup(force_mp, irep) (src/force_sumup.F90:15-593). */
int tis_force_sumup(tis_ctx *ctx, int32_t irep, double *force_mp);

/* No counterpart in the reference.  Neighbour lists and forces of replica
 * irep for caller-owned DEVICE arrays xyz_dev (in) and force_dev (out), each
 * 3*nmp doubles laid out like xyz_mp, without allocating device memory: all
 * per-call scratch comes from one fixed 1 MiB array that every GPU loading
 * the library holds until exit.  It serves hosts whose device memory is held
 * by their own pool allocator, or that must not grow device memory after
 * start-up.  Topology, parameters and the replica's temperature label come
 * from ctx; ctx's own state, lists and flags are untouched.  The scratch of
 * one call is, rounded up to 256-byte blocks, 2 descriptors per replica of
 * ctx + 120 nmp + 8 nmp ceil(nmp/32) + 3 nslot (4 or 8 bytes: mixed or FP64)
 * + 9 nhb + 4 nhbsite bytes, plus 24 nmp + nmp^2 with a periodic box: about
 * 1,700 beads fit without a periodic box and about 840 with one.  Larger
 * replicas, Ewald and Brownian-HI contexts return TIS_E_UNSUPPORTED.  The
 * first call on each device looks up that array's address (set-up) and
 * should come before any stream capture; the address belongs to the
 * device's primary context, so a process that resets the device must not
 * call this afterwards.  All calls on a GPU share the array: calls that
 * overlap on the GPU (other threads, other contexts) race.  Runs on ctx's
 * stream; xyz_dev must be ready when called, force_dev is ready on return.
 * Returns like tis_force_sumup. */
int tis_force_sumup_static(tis_ctx *ctx, int32_t irep, const double *xyz_dev, double *force_dev);

/* energy_sumup(irep, ...) -> energy(E_TYPE%MAX) (src/energy_sumup.F90:11-530). */
int tis_energy_sumup(tis_ctx *ctx, int32_t irep, double *energy);

/* time_integral_pre (src/time_integral_pre.F90:75-180): neighbour lists of
 * every replica, dxyz = 0, forces and a(0) = F/m + rlan_const(1)*xi. */
int tis_time_integral_pre(tis_ctx *ctx);

/* nsteps calls of time_integral (src/time_integral.F90:13-473): neighbour
 * trigger, noise, x update, force_sumup, v/a update, for every replica. */
int tis_step(tis_ctx *ctx, int64_t nsteps);

/* time_integral(flg_step_each_replica) called nsteps times
 * (src/time_integral.F90:13-473 with :134 and :460-465): a replica whose
 * flg_step_each_replica[irep-1] is nonzero on entry does not move; a
 * replica whose step counter reaches exchange_step[irep-1] stops there and
 * gets its flag set (exchange_step(grep) of var_replica, indexed by
 * replica; NULL: no replica stops early).  The caller clears the flags and
 * moves exchange_step on after each exchange, as time_integral_post does
 * (src/time_integral_post.F90:275,363).  Not available on the
 * Brownian-HI path (TIS_E_UNSUPPORTED). */
int tis_time_integral(tis_ctx *ctx, int64_t nsteps, int32_t *flg_step_each_replica,
                      const int64_t *exchange_step);

/* The time-integral loop of mloop_simulator (src/mloop_simulator.F90:
 * 123-150) for replicas that step together: nperiod times [nstep calls of
 * time_integral for every replica; when exchange is nonzero, the replica
 * exchange of time_integral_post (src/time_integral_post.F90:275-363) with
 * counter-based uniforms, as tis_replica_exchange(ctx, NULL, NULL)].  The
 * kernels of one period are recorded once as a CUDA graph on the library's
 * stream (again when nstep or exchange differ from the last call) and
 * replayed, so a period costs one graph launch and no host wait; the host
 * waits once at the end and reports the replicas' errors (NaN, list
 * overflow) of the whole run there; tis_last_step_ms then gives the device
 * time of the last period's steps.  nstep >= 1.  Returns like tis_step.
 * TIS_E_UNSUPPORTED: Brownian-HI contexts, injected noise or uniforms
 * (tis_set_noise), and exchange on a context tis_replica_exchange refuses. */
int tis_run(tis_ctx *ctx, int32_t nperiod, int64_t nstep, int32_t exchange);

/* Step counter (istep) of every replica, istep[nrep]. */
int tis_get_steps(tis_ctx *ctx, int64_t *istep);

/* The Gaussian noise r_boxmuller(3, nmp, nrep) that the library's
 * counter-based generator (Philox4x32-10 with the Box-Muller transform,
 * keyed by seed, replica and step) gives every bead of every replica at
 * steps istep .. istep + nstep - 1, as the reference's get_random_number
 * fills it each step (src/time_integral.F90:121-127); r_boxmuller is
 * (3, nmp_total, nstep).  Injected noise (tis_set_noise) does not affect it. */
int tis_get_random_number(tis_ctx *ctx, int64_t istep, int32_t nstep, double *r_boxmuller);

/* Neighbour rebuilds of replica irep since init and the step of the last
 * one (-1: none): the information of the reference's neighbour-list record
 * (outfile%neigh, src/time_integral.F90:76-84).  Either pointer may be NULL. */
int tis_get_rebuild_info(tis_ctx *ctx, int32_t irep, int64_t *n_rebuild, int64_t *last_step);

/* Replica exchange over temperature labels (src/energy_allrep.F90:123-260 and
 * src/simu_replica_exchange.F90:18-300): energies at the own and the partner
 * label's temperature, Metropolis with uniform u[k] for the k-th pair, label
 * swap and velocity rescale, then the alternation of odd/even pairs.
 * u == NULL draws counter-based uniforms.  n_accept receives the number of
 * accepted swaps. */
int tis_replica_exchange(tis_ctx *ctx, const double *u, int32_t *n_accept);
/* Ladder contexts, step 1 of an exchange: replica_energy(2, nrep_local) of
 * the context's replicas, the energy at the own label and at the exchange
 * partner's label (0 without a partner), as energy_allrep computes it before
 * the ranks gather it (src/energy_allrep.F90:123-217,
 * src/time_integral_post.F90:279).  The caller gathers the ranks' arrays in
 * replica order into replica_energy(2, nrep_all). */
int tis_rex_energies(tis_ctx *ctx, double *replica_energy);

/* Ladder contexts, step 2: the exchange of the whole ladder from the
 * gathered replica_energy(2, nrep_all) (src/simu_replica_exchange.F90:
 * 121-267): every rank takes the same decisions (u == NULL: counter-based
 * uniforms from the shared seed), keeps the ladder's label maps, and
 * relabels and rescales the velocities of its own replicas. */
int tis_rex_exchange_all(tis_ctx *ctx, const double *replica_energy_all, const double *u, int32_t *n_accept);

/* The Metropolis decisions of one exchange of an nrep_all ladder on the host,
 * without a context or a GPU (src/simu_replica_exchange.F90:121-267): pairs
 * of the odd/even alternation idx_pair (1 or 2) in label order, the k-th
 * taking u[k]; rep2lab (1-based, in/out) is updated; vscale[r] (may be NULL)
 * is sqrt(T_new/T_old) for a replica that moved up the ladder, minus it for
 * its partner (whose velocities are divided by it), 0 otherwise. */
int tis_rex_decide(int32_t nrep_all, const double *tempk_all, int32_t idx_pair, const double *replica_energy,
                   const double *u, int32_t *rep2lab, double *vscale, int32_t *n_accept);

/* rep2lab(nrep), 1-based labels. */
int tis_get_labels(tis_ctx *ctx, int32_t *rep2lab);

int tis_status(tis_ctx *ctx, tis_status_t *st);

/* Milliseconds of the last tis_step (or of the steps of tis_run's last
 * period) measured with CUDA events on the library's stream. */
double tis_last_step_ms(tis_ctx *ctx);

/* Device timer on the library's stream: op 0 records the start event; op 1
 * records the stop event, waits for it and writes the elapsed milliseconds
 * to *ms.  Lets a caller time a sequence of library calls on the device. */
int tis_timer(tis_ctx *ctx, int32_t op, double *ms);

/* Human-readable text of the last error on this context. */
const char *tis_last_error(const tis_ctx *ctx);

/* Brownian-HI: diffuse_tensor and random_tensor of replica irep as the last
 * refresh left them (simu_hydro_tensors.F90:17-352; var_simu arrays), each
 * (3 nmp, 3 nmp) column-major; random_tensor is the lower Cholesky factor.
 * Either pointer may be NULL. */
int tis_get_hydro_tensors(tis_ctx *ctx, int32_t irep, double *diffuse, double *random);

/* No counterpart in the reference: number of CUDA kernels this context has
 * launched so far (lets a caller count the launches of a timed region). */
int64_t tis_launch_count(const tis_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* TIS_B200_H */
