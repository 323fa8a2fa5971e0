// api.cu -- host side of the C-ABI (include/tis_b200.h): context set-up,
// temperature-dependent parameters, buffer management and launches.
//
// Host-side parameter set-up restates, in the same FP64 operation order:
//   simu_ele_set.F90:46-226 (dielectric, Bjerrum coefficient, Debye length),
//   simu_set_dtrna.F90:43-58 (stack U0(T), beta_hbond15),
//   time_integral_pre.F90:160-171 (rlan_const), simu_para.F90:26-27,
//   mloop_neigh_dist.F90:28-149, mloop_dtrna.F90:149-152,
//   setp_periodic.F90:78-113, neighbor_list_ele.F90:73-89.
#include <cuda_runtime.h>
#include <algorithm>
#include <array>
#include <map>
#include <cmath>
#include <cstdio>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <dlfcn.h>

#include "../../include/tis_b200.h"
#include "common.cuh"

namespace tis {
size_t smem_bytes_host(int N, int nq, int nslot, int ninc, bool periodic, bool skin, int real_size, int nunit,
                       bool dbuf, int nsite);
cudaError_t lane_kernel_set_smem(bool mixed, int bytes, int bytes2);
cudaError_t lane_kernel_launch_pair(int nlane, size_t smem, cudaStream_t st, const KArgs &a);
size_t smem_base_host(int N, int nq, int nslot, int ninc, bool periodic, bool skin, int real_size, int nunit,
                      bool dbuf);
cudaError_t lane_kernel_launch(bool mixed, int grid, int block, size_t smem, cudaStream_t st, const KArgs &a);
cudaError_t energy_kernel_launch(int grid, int max_nmp, cudaStream_t st, const KArgs &a);
cudaError_t energy_pair_launch(int nlane, int max_nmp, cudaStream_t st, const KArgs &a, const KArgs &b);
cudaError_t noise_launch(cudaStream_t st, KArgs a, long long istep0, int nstep, double *out);
cudaError_t st_status_launch(cudaStream_t st, const KArgs &a, int lane, int nst, int *out);
cudaError_t rex_launch(cudaStream_t st, const KArgs &a, RexState *rex, int *rep2lab, int *lab2rep, int *elabel,
                       double *ebeta);
cudaError_t vscale_launch(cudaStream_t st, const KArgs &a, const double *scale, double *velo);
cudaError_t rex_exchange_launch(cudaStream_t st, const KArgs &a, RexState *rex, int *rep2lab, int *lab2rep,
                                const double *e_own, const double *e_opp, const double *u, double *scale,
                                double *velo);
cudaError_t ewald_recip_launch(cudaStream_t st, const KArgs &a, int nq_max, bool forces);
cudaError_t ewald_energy_launch(cudaStream_t st, const KArgs &a);
cudaError_t bd_refactor_launch(cudaStream_t st, KArgs a, int max_nmp, const int *items, const int *koff);
int bd_refactor_launches(int max_nmp, bool tc);
void bd_update_items(const std::vector<int> &lane_T, std::vector<int> &items, std::vector<int> &koff);
long long bd_plane_floats(int nmp);
cudaError_t bd_step_launch(cudaStream_t st, const KArgs &a, int max_nmp);
cudaError_t bd_force_launch(cudaStream_t st, const KArgs &a, int max_nmp);
}  // namespace tis

using namespace tis;

namespace {

const double F_PI = 3.14159265358979323846264338e0;
const double EPSI_0 = 8.854187817e-12;
const double ELE = 1.6021766208e-19;
const double BOLTZ_J = 1.38064852e-23;
const double N_AVO = 6.022140857e23;
const double KCAL2JOUL = 4184.0;
const double JOUL2KCAL = 1.0 / KCAL2JOUL;
const double JOUL2KCAL_MOL = JOUL2KCAL * N_AVO;
const double BOLTZ_KCAL_MOL = BOLTZ_J * JOUL2KCAL_MOL;

template <typename T> struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  cudaError_t alloc(size_t count) {
    free();
    n = count;
    if (count == 0) count = 1;
    return cudaMalloc((void **)&p, count * sizeof(T));
  }
  cudaError_t upload(const std::vector<T> &v) {
    cudaError_t e = alloc(v.size());
    if (e != cudaSuccess) return e;
    if (!v.empty()) e = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    return e;
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

struct HostTop {   // host copy of one topology with derived tables
  TopDesc d;
  std::vector<int> lunit, uclass;
  std::vector<double> rneigh2;
  int ncharge;
};

}  // namespace

struct tis_ctx {
  tis_params par;
  int nlane = 0, ntop = 0, nlabel = 0;
  int nbead_total = 0;
  int threads = 256, group = 2;
  size_t smem = 0;
  std::vector<TopDesc> tops;
  std::vector<LaneDesc> lanes;
  std::vector<int> lane_nmp;
  std::vector<int> label_top;        // topology of each label
  std::vector<double> lab_T;
  std::vector<int> top_first_label;
  std::vector<int> rep2lab;          // per lane, global label index
  std::vector<int> lab2rep;          // per label, lane
  int idx_pair = 1;                  // odd/even alternation (var_replica.F90:134,165-183)
  int rep_first = 0;                 // ladder context: global replica of lane 0 (irep2grep(1) - 1)
  std::vector<int> g_rep2lab, g_lab2rep;   // ladder context: label maps of the whole ladder (0-based)
  unsigned long long g_counter = 0;  // ladder context: counter of the exchange uniforms
  bool hb_energy_valid = false;      // flg_hb_energy
  double beta_global = 0.0;
  // device buffers
  DBuf<TopDesc> d_tops;
  DBuf<LaneDesc> d_lanes;
  DBuf<LaneState> d_lstate;
  DBuf<int8_t> b_type, b_class;
  DBuf<int16_t> b_unit;
  DBuf<double> b_rcmass, b_cmass, b_fric, b_radius, b_eps, b_charge, b_c2, b_c3, b_c4, b_screen;
  DBuf<int> u_lunit, u_class;
  DBuf<double> rneigh2;
  DBuf<int> bd_idx, ba_idx, st_idx, hb_idx, hb_site, site_val, site_ptr, site_hb, inc_ptr, inc_slot, q_bead;
  DBuf<int> tst_idx, stx_ptr, stx_tst;
  DBuf<double> tst_nat, tst_coef;
  DBuf<double> bd_nat, bd_coef, ba_nat, ba_coef, st_nat, st_coef, hb_nat, hb_coef, hb_nd2;
  DBuf<double> lab_Td, lab_coef, lab_cdist, lab_beta, lab_rele2, lab_u0, lab_c1;
  DBuf<int> lab_u0off, lab_c1off, elabel;
  DBuf<double> xyz, pxyz, velo, accel, dxyz, p0xyz, out_force, out_energy, scale, ebeta;
  DBuf<double> e_opp, rex_u;         // partner energies and injected uniforms of an exchange
  DBuf<int> d_rep2lab, d_lab2rep;    // label maps (the device copy is authoritative)
  DBuf<RexState> rex;
  unsigned long long rex_counter = 0;
  DBuf<uint32_t> mask;
  DBuf<int> site_exc;
  DBuf<uint8_t> mirror, hb_flag;
  DBuf<uint8_t> hb_tert;            // (hb) 1: tertiary ('T') hydrogen bond
  DBuf<uint8_t> b_qkind;            // (bead) 1: phosphate charge -Zp of the label (i_charge = 1)
  DBuf<double> lab_zp, pmf_e, pmf_f; // per label: Zp; Mg-P table (pmf_nbin per label)
  DBuf<double> hb_ene;
  DBuf<uint8_t> hb_flag2;            // hbond scratch of an exchange's partner-label energy pass
  DBuf<double> hb_ene2;
  DBuf<int> site_exc2;
  DBuf<unsigned char> slots;
  DBuf<double> noise, unif;
  DBuf<int> lane_n;                  // per-lane step counts of the last tis_time_integral
  int noise_nsteps = 0, noise_base = 0, n_unif = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, tev0 = nullptr, tev1 = nullptr;
  double last_ms = 0.0;
  std::string err;
  int last_error = 0;
  int wait_timeout = 0, not_spd = 0;
  std::vector<long long> clamp_seen;
  long long launches = 0;            // kernels this context has launched
  bool pair = false;                 // tis_step runs two CTAs (a cluster) per lane
  int noise_sweep = 1, order = 1, sweep = 1, launch_source = 0;
  std::vector<int> h_order;          // launch order of the lanes (order 2: largest first)
  DBuf<int> d_order;
  size_t smem2 = 0;
  // tis_run: the recorded period (nstep steps [+ exchange]) and its launches
  cudaGraphExec_t g_exec = nullptr;
  cudaEvent_t g_ev0 = nullptr, g_ev1 = nullptr;   // recorded around the period's steps
  long long g_nstep = -1, g_launches = 0;
  int g_exchange = -1;
  // Ewald
  int nk = 0, hmax = 0, nqblk = 1, nq_max = 0;
  DBuf<int8_t> ew_h;
  DBuf<double> ew_coef, ew_tab, ew_S, f_ext;
  // Brownian dynamics with hydrodynamic interactions
  bool bdhi = false;
  int max_nmp = 0;
  long long bd_istep = 0;
  DBuf<int> fene_idx, wca_idx, bd_ptr, d_not_spd;
  DBuf<int2> bd_ent;
  DBuf<double> fene_cls, wca_cls, b_hrad;
  DBuf<double> fene_nat, fene_coef, fene_d2, wca_nat, wca_coef, bd_D, bd_L, bd_F, bd_xi;
  DBuf<float> bd_P, bd_D32, bd_L32;
  DBuf<int> bd_items;               // tensor-core update work items, per launch
  std::vector<int> bd_koff;
  DBuf<double> bd_W;
  bool refine = false;               // Brownian-HI: refined noise (tis_params.hi_refine)
  DBuf<double> bd_D64, bd_z;
  DBuf<float> bd_E32, bd_W32;
};

namespace {

int fail(tis_ctx *c, int code, const std::string &msg) {
  if (c) {
    c->err = msg;
    c->last_error = code;
  }
  return code;
}

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(c, TIS_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
  } while (0)

// simu_ele_set.F90:46-226 (i_temp_independent = 0, i_charge = 0)
void ele_params(const tis_params &p, double tempk, double &ek, double &coef, double &cdist) {
  const double MM_A = 87.740e0, MM_B = -0.4008e0, MM_C = 9.398e-4, MM_D = -1.410e-6;
  if (p.i_diele == 0) {
    ek = p.diele_water;
  } else {
    double Tc = tempk - 273.15e0;
    ek = MM_A + MM_B * Tc + MM_C * Tc * Tc + MM_D * Tc * Tc * Tc;
  }
  coef = JOUL2KCAL_MOL * 1.0e10 * (ELE * ELE) / (4.0e0 * F_PI * EPSI_0 * ek);
  cdist = 1.0e10 * std::sqrt((1.0e-3 * EPSI_0 * ek * BOLTZ_J) / (2.0 * N_AVO * (ELE * ELE))) *
          std::sqrt(tempk / p.ionic_strength);
}

// simu_ele_set.F90:107-151: Manning condensation on the phosphates.  The
// DT19 model with Mg balances monovalent and Mg condensation (theta); else
// Zp = b / l_B.  ek is the dielectric constant at temperature tempk.
double manning_zp(const tis_params &p, double tempk, double ek, int n_mg, bool dt19) {
  const double lb = ELE * ELE / (4.0e0 * F_PI * EPSI_0 * ek * BOLTZ_J * tempk) * 1.0e10;
  const double b = p.length_per_unit_P;
  if (!(dt19 && n_mg > 0)) return b / lb;
  const double xi = lb / b, b3 = b * b * b;
  const double conc_Mg = n_mg / (N_AVO * 1.0e-27 * p.psize[0] * p.psize[1] * p.psize[2]);
  const double v1 = 4 * F_PI * b3 * (xi - 1.0e0) * 2;
  const double v2 = 4 * F_PI * b3 * (xi - 0.5e0) * (2 + 1);
  const double c1v1 = (N_AVO * 1.0e-27) * p.ionic_strength * v1;
  const double c2v2 = (N_AVO * 1.0e-27) * conc_Mg * v2;
  const double c1v1_2 = c1v1 * c1v1;
  const double theta =
      (-c1v1_2 + std::sqrt(c1v1_2 * c1v1_2 + 8.0e0 * c1v1_2 * c2v2 * (1.0e0 - 1.0e0 / xi))) / (4.0e0 * c2v2);
  return 1.0 - theta;
}

// simu_ele_set.F90:231-253: Mg-P energy table = PMF, switched to the DH
// energy of charges +2 and -Zp below pmf_rmerge, and its finite-difference
// force; the force of the last point is 0 (the reference never sets it).
// coef is the DH coefficient of the temperature, cdist the Debye length.
void pmf_table(const tis_params &p, double coef, double cdist, double zp, double *e, double *f) {
  const int nb = p.pmf_nbin;
  for (int ib = 0; ib < nb; ++ib) {
    const double r = p.pmf_rmin + p.pmf_rbin * (double)ib;
    const double DH = coef * 2.0 * (-zp) * std::exp(-r / cdist) / r;
    const double e_add = (DH - p.pmf_mg_p[ib]) * std::exp(-(p.pmf_rmerge * p.pmf_rmerge) / (r * r));
    e[ib] = p.pmf_mg_p[ib] + e_add;
  }
  const double rbininv = 1.0 / p.pmf_rbin;
  for (int ib = 0; ib + 1 < nb; ++ib) f[ib] = -rbininv * (e[ib + 1] - e[ib]);
  f[nb - 1] = 0.0;
}

template <typename T>
void append(std::vector<T> &dst, const T *src, size_t n) {
  if (n) dst.insert(dst.end(), src, src + n);
}

// ------------------------------------------------------------ launch configuration
// The step kernel's launch configuration: threads per CTA, threads per bead
// in the force gather, CTAs per replica, where the two-CTA step draws its
// noise, and the launch order of the replicas.  Measured choices come from
// the table the autotuner (tis_b200/autotune.py) writes; each row is a
// workload key and the fastest configuration measured for it:
//   nmp nlane precision i_ele periodic skin | threads group ctas noise_sweep order sweep | rate
// (rows without the sweep column leave it to the built-in rule)
struct LaunchCfg {
  int threads = 0, group = 0, ctas = 0, noise_sweep = 0, order = 0, sweep = 0;
};

struct TuneRow {
  int nmp, nlane, precision, ele, periodic, skin;
  LaunchCfg cfg;
};

std::string library_dir() {
  Dl_info info;
  if (dladdr((void *)&library_dir, &info) && info.dli_fname) {
    const std::string p = info.dli_fname;
    const size_t k = p.rfind('/');
    return k == std::string::npos ? std::string(".") : p.substr(0, k);
  }
  return ".";
}

std::vector<TuneRow> read_tune_table(const std::string &path) {
  std::vector<TuneRow> rows;
  FILE *f = std::fopen(path.c_str(), "r");
  if (!f) return rows;
  char line[512];
  while (std::fgets(line, sizeof line, f)) {
    if (line[0] == '#' || line[0] == '\n') continue;
    TuneRow r{};
    double v[13];
    int n = 0;
    for (char *tok = std::strtok(line, " \t\r\n"); tok && n < 13; tok = std::strtok(nullptr, " \t\r\n"))
      v[n++] = std::atof(tok);
    if (n != 12 && n != 13) continue;   // the rate is the last column
    int *f[12] = {&r.nmp, &r.nlane, &r.precision, &r.ele, &r.periodic, &r.skin, &r.cfg.threads, &r.cfg.group,
                  &r.cfg.ctas, &r.cfg.noise_sweep, &r.cfg.order, &r.cfg.sweep};
    for (int k = 0; k < n - 1; ++k) *f[k] = (int)v[k];
    if (r.nmp > 0 && r.nlane > 0) rows.push_back(r);
  }
  std::fclose(f);
  return rows;
}

// the measured row of the same arithmetic, electrostatics, box and rebuild
// rule nearest in (log nmp, log nlane)
bool tune_lookup(const std::vector<TuneRow> &rows, int nmp, int nlane, int precision, int ele, int periodic, int skin,
                 LaunchCfg &out) {
  double best = 1e300;
  for (int pass = 0; pass < 2 && best == 1e300; ++pass)
    for (const TuneRow &r : rows) {
      if (r.precision != precision || r.ele != ele || r.periodic != periodic) continue;
      if (pass == 0 && r.skin != skin) continue;   // the other rule only when none matches
      const double d = std::fabs(std::log((double)nmp / r.nmp)) + std::fabs(std::log((double)nlane / r.nlane));
      if (d < best) { best = d; out = r.cfg; }
    }
  return best < 1e300;
}

int env_int(const char *name) {
  const char *e = std::getenv(name);
  return e ? std::atoi(e) : 0;
}

// Reciprocal vectors of mloop_ewld.F90:56-156: every integer h != 0 with
// |h| <= hmax in (x, y, z) loop order, comb-sorted by |h|^2 with the
// reference's gap rule, and C(k) = 2 pi / L^3 exp(-k^2 / 4 alpha^2) / k^2
// for k = 2 pi h / L.
void ewald_table(double L, double alpha, double hmax, std::vector<int8_t> &hv, std::vector<double> &coef) {
  const int lmax = (int)std::ceil(hmax);
  const double hmax2 = hmax * hmax;
  std::vector<int> hh;
  std::vector<double> h2;
  for (int ix = -lmax; ix <= lmax; ++ix)
    for (int iy = -lmax; iy <= lmax; ++iy)
      for (int iz = -lmax; iz <= lmax; ++iz) {
        if (ix == 0 && iy == 0 && iz == 0) continue;
        const double r2 = (double)ix * ix + (double)iy * iy + (double)iz * iz;
        if (r2 <= hmax2) { hh.push_back(ix); hh.push_back(iy); hh.push_back(iz); h2.push_back(r2); }
      }
  const int n = (int)h2.size();
  int gap = n;
  bool swapped = false;
  while (gap > 1 || swapped) {
    gap = (gap * 10) / 13;
    if (gap < 1) gap = 1;
    else if (gap == 9 || gap == 10) gap = 11;
    swapped = false;
    for (int i = 0; i + gap < n; ++i)
      if (h2[i] > h2[i + gap]) {
        std::swap(h2[i], h2[i + gap]);
        for (int d = 0; d < 3; ++d) std::swap(hh[3 * i + d], hh[3 * (i + gap) + d]);
        swapped = true;
      }
  }
  const double f = 2.0 * F_PI / L;
  hv.resize(3 * (size_t)n);
  coef.resize(n);
  for (int i = 0; i < n; ++i) {
    for (int d = 0; d < 3; ++d) hv[3 * i + d] = (int8_t)hh[3 * i + d];
    coef[i] = 2.0 * F_PI / (L * L * L) * std::exp(-(f * f) * h2[i] / (4.0 * alpha * alpha)) / ((f * f) * h2[i]);
  }
}

}  // namespace

// --------------------------------------------------------------------- init
namespace {
// the whole ladder of a context that holds only some of its replicas
struct Ladder {
  int nall;
  const double *tempk_all;
  int first;
};

int init_impl(int32_t ntop, const tis_topology *tops, const tis_params *par, const int32_t *nrep,
              const double *tempk, const Ladder *lad, tis_ctx **out) {
  if (!out || !tops || !par || !nrep || (!tempk && !lad) || ntop <= 0) return TIS_E_ARG;
  *out = nullptr;
  tis_ctx *c = new tis_ctx();
  c->par = *par;
  const tis_params &p = *par;
  if (p.i_simulate_type != TIS_SIM_LANGEVIN && p.i_simulate_type != TIS_SIM_BROWNIAN_HI) {
    tis_destroy(c);
    return TIS_E_UNSUPPORTED;
  }
  c->bdhi = p.i_simulate_type == TIS_SIM_BROWNIAN_HI;
  // the Brownian-HI path evaluates FENE and WCA records (the C5 bead chains):
  // no electrostatics, no DT15 or harmonic terms
  if (p.i_ele < TIS_ELE_NONE || p.i_ele > TIS_ELE_COULOMB) { tis_destroy(c); return TIS_E_ARG; }
  if (p.hi_refine != 0 && p.hi_refine != 1) { tis_destroy(c); return TIS_E_ARG; }
  c->refine = c->bdhi && p.precision == TIS_PREC_MIXED && p.hi_refine == 1;
  if (c->bdhi && (p.i_ele != TIS_ELE_NONE || !(p.viscosity > 0.0) || p.i_hydro_tensor < 0 || p.i_hydro_tensor > 4)) {
    tis_destroy(c);
    return TIS_E_UNSUPPORTED;
  }
  // DT19 semi-explicit ions: its Mg-P table lives in the Debye-Hueckel
  // routines (force_ele_DH.F90, energy_ele_DH.F90); Manning charges here
  // feed DH and plain Coulomb
  const bool dt19 = p.i_dtrna_model == 2019;
  if (!(p.i_dtrna_model == 0 || p.i_dtrna_model == 2015 || dt19) || (p.i_charge != 0 && p.i_charge != 1) ||
      (p.i_charge == 1 && !(p.length_per_unit_P > 0.0))) {
    tis_destroy(c);
    return TIS_E_ARG;
  }
  if ((dt19 && p.i_ele != TIS_ELE_DH) || (p.i_charge == 1 && p.i_ele == TIS_ELE_EWALD) || (dt19 && c->bdhi)) {
    tis_destroy(c);
    return TIS_E_UNSUPPORTED;
  }
  int n_mg_any = 0;
  for (int k = 0; k < ntop; ++k)
    for (int i = 0; i < tops[k].nmp; ++i) n_mg_any += tops[k].imp2type[i] == TIS_MP_ION_MG;
  // simu_ele_set.F90:231-236: the semi-explicit model with Mg needs i_charge
  // = 1, the table (setp_pmf.F90) and the box that gives [Mg]
  if (dt19 && n_mg_any > 0 &&
      (p.i_charge != 1 || !p.pmf_mg_p || p.pmf_nbin < 2 || !(p.pmf_rbin > 0.0) || !(p.pmf_rmax >= p.pmf_rmin) ||
       !(p.pmf_rmin > 0.0) || p.i_periodic != 1 || !(p.psize[0] * p.psize[1] * p.psize[2] > 0.0))) {
    tis_destroy(c);
    return TIS_E_ARG;
  }
  if (p.i_ele == TIS_ELE_EWALD) {
    // mloop_ewld.F90 uses psize(1) for a cubic box; the per-charge tables
    // hold |h| <= 11
    if (p.i_periodic != 1 || p.psize[0] != p.psize[1] || p.psize[0] != p.psize[2] || !(p.ewld_hmax > 0.0) ||
        std::ceil(p.ewld_hmax) > 11.0 || !(p.ewld_alpha > 0.0)) {
      tis_destroy(c);
      return TIS_E_UNSUPPORTED;
    }
  }
  const bool periodic = p.i_periodic == 1;
  const bool skin = p.n_step_neighbor <= 0;
  c->ntop = ntop;
  // ---- topology tables
  std::vector<int8_t> b_type, b_class;
  std::vector<int16_t> b_unit;
  std::vector<double> b_rcmass, b_cmass, b_fric, b_radius, b_eps, b_charge, b_c2, b_c3, b_c4, b_screen;
  std::vector<int> u_lunit, u_class;
  std::vector<double> rneigh2;
  std::vector<int> bd_idx, ba_idx, st_idx, hb_idx, hb_site, site_val, site_ptr, site_hb, inc_ptr, inc_slot, q_bead;
  std::vector<double> bd_nat, bd_coef, ba_nat, ba_coef, st_nat, st_coef, hb_nat, hb_coef, hb_nd2;
  std::vector<double> st_hsTm_all;
  std::vector<uint8_t> hb_tert;
  bool any_tert = false;
  std::vector<uint8_t> b_qkind;
  std::vector<int> top_nmg(ntop, 0);
  std::vector<int> tst_idx, stx_ptr, stx_tst;
  std::vector<double> tst_nat, tst_coef;
  std::vector<int> fene_idx, wca_idx, bdp;
  std::vector<int2> bde;
  std::vector<double> fene_cls, wca_cls;
  std::map<std::array<double, 3>, int> fene_cmap, wca_cmap;
  std::vector<double> fene_nat, fene_coef, fene_d2, wca_nat, wca_coef;
  std::vector<double> b_hrad;   // Brownian-HI: hydrodynamic radius of every bead
  int maxN = 0;
  for (int k = 0; k < ntop; ++k) {
    const tis_topology &t = tops[k];
    if (t.nmp <= 0 || t.nmp > 65535 || t.nunit <= 0) { tis_destroy(c); return TIS_E_ARG; }
    TopDesc d{};
    d.nmp = t.nmp;
    d.nunit = t.nunit;
    d.bead0 = (int)b_type.size();
    d.unit0 = (int)u_class.size();
    d.rn0 = (int)rneigh2.size();
    d.bd0 = (int)bd_nat.size(); d.nbd = t.nbd;
    d.ba0 = (int)ba_nat.size(); d.nba = t.nba;
    d.st0 = (int)(st_nat.size() / 3); d.nst = t.nst;
    d.tst0 = (int)(tst_nat.size() / 6); d.ntst = t.ntst;
    d.stx0 = (int)stx_ptr.size();
    d.hb0 = (int)(hb_nat.size() / 6); d.nhb = t.nhb;
    d.site0 = (int)site_val.size(); d.nsite = t.nhbsite;
    d.sitehb0 = (int)site_hb.size();
    d.inc0 = (int)inc_ptr.size();
    d.slot_ba = 2 * t.nbd;
    d.slot_st = d.slot_ba + 3 * t.nba;
    d.slot_tst = d.slot_st + 7 * t.nst;
    d.slot_hb = d.slot_tst + 6 * t.ntst;
    d.nslot = d.slot_hb + 6 * t.nhb;
    maxN = std::max(maxN, t.nmp);
    if (c->bdhi && (t.nbd || t.nba || t.nst || t.nhb || t.ntst)) { tis_destroy(c); return TIS_E_UNSUPPORTED; }
    // FENE / WCA records (read_nativeinfo.F90:153-176, 306-332); per bead
    // incidence lists for the Brownian-HI force gather, FENE records first:
    // (partner bead, parameter class * 2 + kind), classes = the distinct
    // parameter triples
    d.fe0 = (int)fene_nat.size(); d.nfe = t.nfene;
    d.wc0 = (int)wca_nat.size(); d.nwc = t.nwca;
    d.bp0 = (int)bdp.size(); d.be0 = (int)bde.size();
    if (c->bdhi) {
      for (int i = 0; i < t.nmp; ++i) {
        const double r = t.radius ? t.radius[i] : p.hi_radius;
        if (!(r > 0.0)) { tis_destroy(c); return TIS_E_ARG; }
        b_hrad.push_back(r);
      }
      std::vector<std::vector<int2>> per(t.nmp);
      auto cls_of = [](std::map<std::array<double, 3>, int> &m, std::vector<double> &tab, double p0, double p1,
                       double p2) {
        const std::array<double, 3> key{p0, p1, p2};
        auto it = m.find(key);
        if (it != m.end()) return it->second;
        const int id = (int)m.size();
        m.emplace(key, id);
        tab.push_back(p0); tab.push_back(p1); tab.push_back(p2);
        return id;
      };
      for (int r = 0; r < t.nfene; ++r) {
        const int i1 = t.ifene2mp[2 * r] - 1, i2 = t.ifene2mp[2 * r + 1] - 1;
        if (i1 < 0 || i2 < 0 || i1 >= t.nmp || i2 >= t.nmp || i1 == i2) { tis_destroy(c); return TIS_E_ARG; }
        fene_idx.push_back(i1); fene_idx.push_back(i2);
        fene_nat.push_back(t.fene_nat[r]); fene_coef.push_back(t.coef_fene[r]); fene_d2.push_back(t.dist2_fene[r]);
        const int cl = cls_of(fene_cmap, fene_cls, t.fene_nat[r], t.coef_fene[r], t.dist2_fene[r]);
        per[i1].push_back(make_int2(i2, 2 * cl)); per[i2].push_back(make_int2(i1, 2 * cl));
      }
      for (int r = 0; r < t.nwca; ++r) {
        const int i1 = t.iwca2mp[2 * r] - 1, i2 = t.iwca2mp[2 * r + 1] - 1;
        if (i1 < 0 || i2 < 0 || i1 >= t.nmp || i2 >= t.nmp || i1 == i2) { tis_destroy(c); return TIS_E_ARG; }
        wca_idx.push_back(i1); wca_idx.push_back(i2);
        wca_nat.push_back(t.wca_nat[r]);
        wca_coef.push_back(t.coef_wca[r]); wca_coef.push_back(t.coef_wca[t.nwca + r]);
        const int cl = cls_of(wca_cmap, wca_cls, t.wca_nat[r], t.coef_wca[r], t.coef_wca[t.nwca + r]);
        per[i1].push_back(make_int2(i2, 2 * cl + 1)); per[i2].push_back(make_int2(i1, 2 * cl + 1));
      }
      int off = 0;
      for (int i = 0; i < t.nmp; ++i) {
        bdp.push_back(off);
        for (const int2 &e : per[i]) bde.push_back(e);
        off += (int)per[i].size();
      }
      bdp.push_back(off);
    }
    // beads
    std::vector<int> imp2unit(t.nmp, 0);
    for (int u = 0; u < t.nunit; ++u) {
      int a0 = t.lunit2mp[2 * u] - 1, a1 = t.lunit2mp[2 * u + 1] - 1;
      if (a0 < 0 || a1 >= t.nmp || a1 < a0) { tis_destroy(c); return TIS_E_ARG; }
      for (int i = a0; i <= a1; ++i) imp2unit[i] = u;
      u_lunit.push_back(a0);
      u_lunit.push_back(a1);
      u_class.push_back(t.iclass_unit[u]);
    }
    std::vector<double> q(t.nmp, 0.0);
    std::vector<uint8_t> qk(t.nmp, 0);
    for (int i = 0; i < t.ncharge; ++i) {
      const int b = t.icharge2mp[i] - 1;
      if (b < 0 || b >= t.nmp) { tis_destroy(c); return TIS_E_ARG; }
      q[b] = t.coef_charge[i];
      // simu_ele_set.F90:150-166: with i_charge = 1 every phosphate that no
      // CHARGE_CHANGE line fixes carries -Zp of its temperature (Zp > 0)
      if (p.i_charge == 1 && t.imp2type[b] == TIS_MP_RNA_PHOS && !(t.flg_charge_fixed && t.flg_charge_fixed[i]))
        qk[b] = 1;
    }
    for (int i = 0; i < t.nmp; ++i) top_nmg[k] += t.imp2type[i] == TIS_MP_ION_MG;
    // charged beads in icharge order (neighbor_list_ele.F90:126,138 skip |q| < ZERO_JUDGE)
    d.q0 = (int)q_bead.size();
    for (int i = 0; i < t.ncharge; ++i) {
      if (i > 0 && t.icharge2mp[i] <= t.icharge2mp[i - 1]) { tis_destroy(c); return TIS_E_ARG; }
      if (qk[t.icharge2mp[i] - 1] || std::fabs(t.coef_charge[i]) >= 1.0e-6) q_bead.push_back(t.icharge2mp[i] - 1);
    }
    d.nq = (int)q_bead.size() - d.q0;
    for (int i = 0; i < t.nmp; ++i) {
      b_type.push_back((int8_t)t.imp2type[i]);
      b_class.push_back((int8_t)t.iclass_unit[imp2unit[i]]);
      b_unit.push_back((int16_t)imp2unit[i]);
      b_cmass.push_back(t.cmass[i]);
      b_rcmass.push_back(1.0e0 / t.cmass[i]);
      b_fric.push_back(t.fric[i]);
      b_radius.push_back(t.exv_radius[i]);
      b_eps.push_back(t.exv_epsilon[i]);
      b_charge.push_back(q[i]);
      b_qkind.push_back(qk[i]);
      // time_integral_pre.F90:162-170
      double tfh = 0.5e0 * p.tstep * t.fric[i];
      double u1 = 1.0e0 - tfh;
      double u2 = 1.0e0 - tfh + tfh * tfh;
      b_c2.push_back(u1 * u2);
      b_c3.push_back((0.5e0 * p.tstep) * u1);
      b_c4.push_back(p.tstep * u1);
    }
    // exv screen radius: the largest contact distance dij the bead can have
    // (force_exv_dt15.F90:220-228): RNA-RNA pairs use exv_dist / exv_dist_PS,
    // every other pair the sum of the two radii
    {
      double rmax_all = 0.0, rmax_non_rna = 0.0;
      for (int i = 0; i < t.nmp; ++i) {
        rmax_all = std::max(rmax_all, t.exv_radius[i]);
        if (t.iclass_unit[imp2unit[i]] != TIS_CLASS_RNA) rmax_non_rna = std::max(rmax_non_rna, t.exv_radius[i]);
      }
      for (int i = 0; i < t.nmp; ++i) {
        double sc;
        if (dt19)   // force_exv_dt15.F90:60-66: base-base exv_dist, every other pair the radius sum
          sc = std::max(p.exv_dist, t.exv_radius[i] + rmax_all);
        else if (t.iclass_unit[imp2unit[i]] == TIS_CLASS_RNA)
          sc = std::max(std::max(p.exv_dist, p.exv_dist_PS), rmax_non_rna > 0 ? t.exv_radius[i] + rmax_non_rna : 0.0);
        else
          sc = t.exv_radius[i] + rmax_all;
        b_screen.push_back(sc);
      }
    }
    // mloop_neigh_dist.F90:28-149
    for (int u = 0; u < t.nunit; ++u)
      for (int v = 0; v < t.nunit; ++v) {
        double max_cut = 0.0;
        if (t.iclass_unit[u] == TIS_CLASS_RNA && t.iclass_unit[v] == TIS_CLASS_RNA) {
          if (p.exv_dist > max_cut) max_cut = p.exv_dist;
          if (p.exv_dist_PS > max_cut) max_cut = p.exv_dist_PS;
        } else {
          for (int i = t.lunit2mp[2 * u] - 1; i <= t.lunit2mp[2 * u + 1] - 1; ++i)
            for (int j = t.lunit2mp[2 * v] - 1; j <= t.lunit2mp[2 * v + 1] - 1; ++j) {
              double cut = t.exv_radius[i] + t.exv_radius[j];
              if (cut > max_cut) max_cut = cut;
            }
        }
        double r = max_cut + p.neigh_margin;
        rneigh2.push_back(r * r);
      }
    for (int i = 0; i < 2 * t.nbd; ++i) bd_idx.push_back(t.ibd2mp[i] - 1);
    append(bd_nat, t.bd_nat, t.nbd);
    append(bd_coef, t.coef_bd, t.nbd);
    for (int i = 0; i < 3 * t.nba; ++i) ba_idx.push_back(t.iba2mp[i] - 1);
    append(ba_nat, t.ba_nat, t.nba);
    append(ba_coef, t.coef_ba, t.nba);
    for (int i = 0; i < 7 * t.nst; ++i) st_idx.push_back(t.idtrna_st2mp[i] - 1);
    append(st_nat, t.dtrna_st_nat, 3 * (size_t)t.nst);
    append(st_coef, t.coef_dtrna_st, 3 * (size_t)t.nst);
    append(st_hsTm_all, t.dtrna_st_hsTm, 3 * (size_t)t.nst);
    // tertiary stacks; each side's secondary stack (mloop_dtrna.F90:74-140):
    // the stack of base B with B - 3 (side 1) or B + 3 (side 2), exclusive
    // only when that stack exists; per secondary stack the list of the
    // tertiary stacks that can turn it off
    {
      std::vector<std::vector<int>> excl(t.nst);
      for (int i = 0; i < 6 * t.ntst; ++i) {
        if (t.idtrna_tst2mp[i] < 1 || t.idtrna_tst2mp[i] > t.nmp) { tis_destroy(c); return TIS_E_ARG; }
        tst_idx.push_back(t.idtrna_tst2mp[i] - 1);
      }
      append(tst_nat, t.dtrna_tst_nat, 6 * (size_t)t.ntst);
      append(tst_coef, t.coef_dtrna_tst, 7 * (size_t)t.ntst);
      for (int itst = 0; itst < t.ntst; ++itst)
        for (int sd = 0; sd < 2; ++sd) {
          const int imp1 = t.idtrna_tst2mp[6 * itst + sd];
          const int side = t.idtrna_tst2side[2 * itst + sd];
          if (side != 1 && side != 2) { tis_destroy(c); return TIS_E_ARG; }
          const int imp2 = side == 1 ? imp1 - 3 : imp1 + 3;
          for (int ist = 0; ist < t.nst; ++ist) {
            const int a1 = t.idtrna_st2mp[7 * ist], a2 = t.idtrna_st2mp[7 * ist + 1];
            if ((imp1 == a1 && imp2 == a2) || (imp1 == a2 && imp2 == a1)) {
              if (t.flg_tst_exclusive[2 * itst + sd]) excl[ist].push_back(itst);
              break;
            }
          }
        }
      if (t.ntst > 0) {
        int off = (int)stx_tst.size();
        for (int ist = 0; ist < t.nst; ++ist) {
          stx_ptr.push_back(off);
          for (int e : excl[ist]) stx_tst.push_back(e);
          off += (int)excl[ist].size();
        }
        stx_ptr.push_back(off);
      }
    }
    for (int i = 0; i < 6 * t.nhb; ++i) hb_idx.push_back(t.idtrna_hb2mp[i] - 1);
    append(hb_nat, t.dtrna_hb_nat, 6 * (size_t)t.nhb);
    append(hb_coef, t.coef_dtrna_hb, 7 * (size_t)t.nhb);
    for (int i = 0; i < 6 * t.nhb; ++i) hb_site.push_back(t.idtrna_hb2hbsite[i] - 1);
    for (int h = 0; h < t.nhb; ++h) {   // read_nativeinfo.F90:606-613
      const uint8_t tt = (t.flg_hb_tertiary && t.flg_hb_tertiary[h]) ? 1 : 0;
      hb_tert.push_back(tt);
      any_tert = any_tert || tt;
    }
    for (int h = 0; h < t.nhb; ++h) {   // mloop_dtrna.F90:151
      double r = t.dtrna_hb_nat[6 * h] + p.hb_cutoff_dist + p.neigh_margin;
      hb_nd2.push_back(r * r);
    }
    for (int s = 0; s < t.nhbsite; ++s) site_val.push_back(t.nvalence_hbsite[s]);
    // per-site hbond lists in list_hb_at_hbsite order (neighbor_list_hb.F90:394-410)
    std::vector<std::vector<int>> at(t.nhbsite);
    for (int h = 0; h < t.nhb; ++h)
      for (int i = 0; i < 3; ++i) {
        int s1 = t.idtrna_hb2hbsite[6 * h + i], s2 = t.idtrna_hb2hbsite[6 * h + 3 + i];
        if (s1 > 0) at[s1 - 1].push_back(h);
        if (s2 > 0) at[s2 - 1].push_back(h);
      }
    int cnt = 0;
    for (int s = 0; s < t.nhbsite; ++s) {
      site_ptr.push_back(cnt);
      for (int h : at[s]) site_hb.push_back(h);
      cnt += (int)at[s].size();
    }
    site_ptr.push_back(cnt);
    // incidence lists: bead -> slots, ascending slot id
    std::vector<std::vector<int>> inc(t.nmp);
    for (int b = 0; b < t.nbd; ++b)
      for (int q2 = 0; q2 < 2; ++q2) inc[t.ibd2mp[2 * b + q2] - 1].push_back(2 * b + q2);
    for (int b = 0; b < t.nba; ++b)
      for (int q2 = 0; q2 < 3; ++q2) inc[t.iba2mp[3 * b + q2] - 1].push_back(d.slot_ba + 3 * b + q2);
    for (int b = 0; b < t.nst; ++b)
      for (int q2 = 0; q2 < 7; ++q2) inc[t.idtrna_st2mp[7 * b + q2] - 1].push_back(d.slot_st + 7 * b + q2);
    for (int b = 0; b < t.ntst; ++b)
      for (int q2 = 0; q2 < 6; ++q2) inc[t.idtrna_tst2mp[6 * b + q2] - 1].push_back(d.slot_tst + 6 * b + q2);
    for (int b = 0; b < t.nhb; ++b)
      for (int q2 = 0; q2 < 6; ++q2) inc[t.idtrna_hb2mp[6 * b + q2] - 1].push_back(d.slot_hb + 6 * b + q2);
    int ip = (int)inc_slot.size();
    const int ip0 = ip;
    for (int i = 0; i < t.nmp; ++i) {
      inc_ptr.push_back(ip);
      for (int sl : inc[i]) inc_slot.push_back(sl);
      ip += (int)inc[i].size();
    }
    inc_ptr.push_back(ip);
    d.ninc = ip - ip0;
    c->tops.push_back(d);
  }
  // ---- labels (temperatures) and lanes (replicas).  Normally lane l starts
  // with label l; a ladder context holds labels for the whole ladder and
  // lanes for its share of the replicas (lane l is global replica first + l)
  int nlane = 0;
  for (int k = 0; k < ntop; ++k) {
    if (nrep[k] <= 0) { tis_destroy(c); return TIS_E_ARG; }
    nlane += nrep[k];
  }
  const int nlabel = lad ? lad->nall : nlane;
  const double *lab_temp = lad ? lad->tempk_all : tempk;
  c->nlane = nlane;
  c->nlabel = nlabel;
  c->rep_first = lad ? lad->first : 0;
  std::vector<double> lab_T(nlabel), lab_coef(nlabel), lab_cdist(nlabel), lab_beta(nlabel), lab_rele2(nlabel);
  std::vector<double> lab_zp(nlabel, 0.0), pmf_e, pmf_f;
  const bool pmf_on = dt19 && n_mg_any > 0;
  if (pmf_on) { pmf_e.assign((size_t)nlabel * p.pmf_nbin, 0.0); pmf_f.assign((size_t)nlabel * p.pmf_nbin, 0.0); }
  std::vector<int> lab_u0off(nlabel), lab_c1off(nlabel);
  std::vector<double> lab_u0, lab_c1;
  c->label_top.resize(nlabel);
  c->rep2lab.resize(nlane);
  c->lab2rep.resize(nlabel);
  {
    int label = 0;
    for (int k = 0; k < ntop; ++k) {
      TopDesc &d = c->tops[k];
      d.nlabel = lad ? nlabel : nrep[k];
      c->top_first_label.push_back(label);
      const int N = d.nmp;
      for (int r = 0; r < d.nlabel; ++r, ++label) {
        const double T = lab_temp[label];
        double ek, coef, cdist;
        ele_params(p, T, ek, coef, cdist);
        lab_T[label] = T;
        lab_coef[label] = coef;
        lab_cdist[label] = cdist;
        if (p.i_charge == 1) lab_zp[label] = manning_zp(p, T, ek, top_nmg[k], dt19);
        if (pmf_on && top_nmg[k] > 0)
          pmf_table(p, coef, cdist, lab_zp[label], &pmf_e[(size_t)label * p.pmf_nbin],
                    &pmf_f[(size_t)label * p.pmf_nbin]);
        lab_beta[label] = 1.0e0 / (T * BOLTZ_KCAL_MOL);
        double rr = (p.i_ele == TIS_ELE_DH) ? (p.neigh_margin + p.cutoff_ele * cdist) : (p.neigh_margin + p.cutoff_ele);
        lab_rele2[label] = rr * rr;
        lab_u0off[label] = (int)lab_u0.size();
        for (int s = 0; s < d.nst; ++s) {   // simu_set_dtrna.F90:48-53
          const double *hst = &st_hsTm_all[3 * (size_t)(d.st0 + s)];
          lab_u0.push_back(-hst[0] + BOLTZ_KCAL_MOL * (T - hst[2]) * hst[1]);
        }
        lab_c1off[label] = (int)lab_c1.size();
        for (int i = 0; i < N; ++i) {   // time_integral_pre.F90:166-167
          const int b = d.bead0 + i;
          lab_c1.push_back(std::sqrt(2.0e0 * b_fric[b] * BOLTZ_KCAL_MOL * T / (p.tstep * b_cmass[b])));
        }
        c->label_top[label] = k;
        c->lab2rep[label] = label;
      }
    }
  }
  size_t mask_off = 0, slot_off = 0;
  long long mirror_off = 0;
  int hb_off = 0, site_off = 0, state_off = 0, ew_off = 0;
  long long bd_off = 0, bdp_off = 0, bd32_off = 0, bdw_off = 0;
  int lane = 0;
  for (int k = 0; k < ntop; ++k) {
    TopDesc &d = c->tops[k];
    const int N = d.nmp;
    for (int r = 0; r < nrep[k]; ++r, ++lane) {
      const int grep = c->rep_first + lane;   // global replica (0-based)
      c->rep2lab[lane] = grep;
      LaneDesc L{};
      L.top = k;
      L.state0 = state_off;
      L.mask0 = (int)mask_off;
      L.mirror0 = mirror_off;
      L.slot0 = (int)slot_off;
      L.hb0 = hb_off;
      L.site0 = site_off;
      L.unif0 = 0;
      L.ew0 = ew_off;
      ew_off += d.nq;
      L.bd0 = bd_off;
      L.bdp0 = bdp_off;
      L.bd32 = bd32_off;
      L.key_lane = grep;
      L.key_bead0 = lad ? grep * N : state_off;
      if (c->bdhi) bd_off += 9LL * N * N;
      L.bdw0 = bdw_off;
      if (c->bdhi && p.precision == TIS_PREC_MIXED) {
        bdp_off += bd_plane_floats(N);
        bd32_off += 3LL * N * ((3LL * N + 3) / 4 * 4);
        if (p.hi_refine == 1) bdw_off += (long long)((3 * N + 63) / 64) * 64 * 64;
      }
      state_off += N;
      mask_off += 2 * (size_t)N * ((N + 31) / 32);
      if (periodic) mirror_off += (long long)N * N;
      slot_off += d.nslot;
      hb_off += d.nhb;
      site_off += d.nsite;
      c->lanes.push_back(L);
      c->lane_nmp.push_back(N);
    }
  }
  if (mask_off > 0x7fffffffULL || slot_off > 0x7fffffffULL) {
    tis_destroy(c);
    return TIS_E_ARG;
  }
  c->nbead_total = state_off;
  c->lab_T = lab_T;
  // the global beta_hbond15 is the value set for the last replica (simu_set_dtrna.F90:58)
  c->beta_global = lab_beta[nlabel - 1];
  if (lad) {
    c->g_rep2lab.resize(nlabel);
    c->g_lab2rep.resize(nlabel);
    for (int g = 0; g < nlabel; ++g) { c->g_rep2lab[g] = g; c->g_lab2rep[g] = g; }
  }
  const int real_size = (p.precision == TIS_PREC_MIXED) ? 4 : 8;
  size_t smem = 0, smem2 = 0;
  int minN = 1 << 30;
  bool pair_fits = true;
  for (auto &d : c->tops) {
    // electrostatic row chunks: one per charged bead at least
    if (p.i_ele != TIS_ELE_NONE && d.nq > CHMAX) { tis_destroy(c); return TIS_E_UNSUPPORTED; }
    c->nq_max = std::max(c->nq_max, d.nq);
    // the per-lane base layout must fit one CTA's shared memory (the
    // Brownian-HI path does not run the lane kernel)
    if (c->bdhi) continue;
    if (smem_base_host(d.nmp, d.nq, d.nslot, d.ninc, periodic, skin, real_size, d.nunit, false) + 64 > 227 * 1024) {
      tis_destroy(c);
      return TIS_E_UNSUPPORTED;
    }
    smem = std::max(smem, smem_bytes_host(d.nmp, d.nq, d.nslot, d.ninc, periodic, skin, real_size, d.nunit, false,
                                          d.nsite));
    smem2 = std::max(smem2, smem_bytes_host(d.nmp, d.nq, d.nslot, d.ninc, periodic, skin, real_size, d.nunit, true,
                                            d.nsite));
    minN = std::min(minN, d.nmp);
    // the two-CTA layout (next-step copies of the positions) must fit too
    if (smem_base_host(d.nmp, d.nq, d.nslot, d.ninc, periodic, skin, real_size, d.nunit, true) + 64 > 227 * 1024)
      pair_fits = false;
  }
  c->smem = smem;
  // launch configuration: caller fields, then the environment, then the
  // tuned table, then the built-in rule (one CTA per replica up to 96 beads
  // on 128 threads, 256 up to 160, else 512; two CTAs per replica when the
  // replicas fill at most half of the SMs; largest replica first in batches)
  {
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const bool mixed = p.precision == TIS_PREC_MIXED;
    const bool pair_ok = !c->bdhi && mixed && !periodic && p.i_ele != TIS_ELE_EWALD && minN >= 64 && pair_fits;
    LaunchCfg cfg;
    int source = 0;
    {
      const std::string path = p.launch_table ? std::string(p.launch_table) : library_dir() + "/tuned_launch.tsv";
      const std::vector<TuneRow> rows = read_tune_table(path);
      if (!c->bdhi && tune_lookup(rows, maxN, nlane, mixed ? 1 : 0, p.i_ele, periodic ? 1 : 0, skin ? 1 : 0, cfg))
        source = 1;
    }
    const int env_t = env_int("TIS_THREADS"), env_g = env_int("TIS_GROUP");
    const char *env_c = std::getenv("TIS_CLUSTER"), *env_n = std::getenv("TIS_NOISE_SWEEP");
    if (env_t) { cfg.threads = env_t; source = 2; }
    if (env_g) { cfg.group = env_g; source = 2; }
    if (env_c) { cfg.ctas = env_c[0] == '0' ? 1 : 2; source = 2; }
    if (env_n) { cfg.noise_sweep = env_n[0] == '0' ? 2 : 1; source = 2; }
    if (p.launch_threads) { cfg.threads = p.launch_threads; source = 2; }
    if (p.launch_group) { cfg.group = p.launch_group; source = 2; }
    if (p.launch_ctas) { cfg.ctas = p.launch_ctas; source = 2; }
    if (p.launch_noise_sweep) { cfg.noise_sweep = p.launch_noise_sweep; source = 2; }
    if (p.launch_order) { cfg.order = p.launch_order; source = 2; }
    if (p.launch_sweep) { cfg.sweep = p.launch_sweep; source = 2; }
    if (cfg.ctas == 0) cfg.ctas = (pair_ok && nsm > 0 && 2 * nlane <= nsm) ? 2 : 1;
    if (cfg.ctas == 2 && !pair_ok) cfg.ctas = 1;
    if (cfg.ctas == 2) cfg.threads = 512;   // the cluster kernel runs 512 threads per CTA
    if (cfg.threads == 0) cfg.threads = maxN <= 96 ? 128 : (maxN <= 160 ? 256 : 512);
    if (cfg.threads < 64 || cfg.threads > (mixed ? 1024 : 512) || cfg.threads % 32) {
      tis_destroy(c);
      return TIS_E_ARG;
    }
    if (!(cfg.group == 0 || cfg.group == 1 || cfg.group == 2 || cfg.group == 4 || cfg.group == 8)) {
      tis_destroy(c);
      return TIS_E_ARG;
    }
    if (cfg.noise_sweep == 0) cfg.noise_sweep = 1;
    if (cfg.order == 0) cfg.order = ntop > 1 ? 2 : 1;
    if (cfg.ctas == 2) cfg.sweep = 1;   // the cluster kernel deals its chunks snake-wise
    else if (cfg.sweep == 0) cfg.sweep = cfg.threads >= 1024 ? 3 : 1;
    if (cfg.sweep < 1 || cfg.sweep > 3) {
      tis_destroy(c);
      return TIS_E_ARG;
    }
    c->threads = cfg.threads;
    c->group = cfg.group;
    c->pair = cfg.ctas == 2;
    c->noise_sweep = cfg.noise_sweep;
    c->order = cfg.order;
    c->sweep = cfg.sweep;
    c->launch_source = source;
    c->smem2 = c->pair ? smem2 : 0;
    // replicas largest first: a CTA that frees its SM takes the next one
    std::vector<int> order(nlane);
    for (int l = 0; l < nlane; ++l) order[l] = l;
    if (c->order == 2)
      std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return c->lane_nmp[x] > c->lane_nmp[y]; });
    c->h_order = order;
  }

  // ---- device
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&c->ev0));
  CK(cudaEventCreate(&c->ev1));
  if (!c->bdhi) CK(lane_kernel_set_smem(p.precision == TIS_PREC_MIXED, (int)smem, (int)c->smem2));
  CK(c->d_order.upload(c->h_order));
  CK(c->d_tops.upload(c->tops));
  CK(c->d_lanes.upload(c->lanes));
  std::vector<LaneState> ls(nlane);
  for (int i = 0; i < nlane; ++i) {
    std::memset(&ls[i], 0, sizeof(LaneState));
    ls[i].label = c->rep2lab[i];
    ls[i].last_rebuild = -1;
  }
  CK(c->d_lstate.upload(ls));
  CK(c->b_type.upload(b_type)); CK(c->b_class.upload(b_class)); CK(c->b_unit.upload(b_unit));
  CK(c->b_rcmass.upload(b_rcmass)); CK(c->b_cmass.upload(b_cmass)); CK(c->b_fric.upload(b_fric));
  CK(c->b_radius.upload(b_radius)); CK(c->b_eps.upload(b_eps)); CK(c->b_charge.upload(b_charge));
  CK(c->b_c2.upload(b_c2)); CK(c->b_c3.upload(b_c3)); CK(c->b_c4.upload(b_c4)); CK(c->b_screen.upload(b_screen));
  CK(c->u_lunit.upload(u_lunit)); CK(c->u_class.upload(u_class)); CK(c->rneigh2.upload(rneigh2));
  CK(c->bd_idx.upload(bd_idx)); CK(c->bd_nat.upload(bd_nat)); CK(c->bd_coef.upload(bd_coef));
  CK(c->ba_idx.upload(ba_idx)); CK(c->ba_nat.upload(ba_nat)); CK(c->ba_coef.upload(ba_coef));
  CK(c->st_idx.upload(st_idx)); CK(c->st_nat.upload(st_nat)); CK(c->st_coef.upload(st_coef));
  CK(c->tst_idx.upload(tst_idx)); CK(c->tst_nat.upload(tst_nat)); CK(c->tst_coef.upload(tst_coef));
  CK(c->stx_ptr.upload(stx_ptr)); CK(c->stx_tst.upload(stx_tst));
  CK(c->hb_idx.upload(hb_idx)); CK(c->hb_nat.upload(hb_nat)); CK(c->hb_coef.upload(hb_coef));
  CK(c->hb_site.upload(hb_site)); CK(c->hb_nd2.upload(hb_nd2));
  if (any_tert) CK(c->hb_tert.upload(hb_tert));
  if (p.i_charge == 1) { CK(c->b_qkind.upload(b_qkind)); CK(c->lab_zp.upload(lab_zp)); }
  if (pmf_on) { CK(c->pmf_e.upload(pmf_e)); CK(c->pmf_f.upload(pmf_f)); }
  CK(c->site_val.upload(site_val)); CK(c->site_ptr.upload(site_ptr)); CK(c->site_hb.upload(site_hb));
  CK(c->inc_ptr.upload(inc_ptr)); CK(c->inc_slot.upload(inc_slot)); CK(c->q_bead.upload(q_bead));
  CK(c->lab_Td.upload(lab_T)); CK(c->lab_coef.upload(lab_coef)); CK(c->lab_cdist.upload(lab_cdist));
  CK(c->lab_beta.upload(lab_beta)); CK(c->lab_rele2.upload(lab_rele2));
  CK(c->lab_u0off.upload(lab_u0off)); CK(c->lab_u0.upload(lab_u0));
  CK(c->lab_c1off.upload(lab_c1off)); CK(c->lab_c1.upload(lab_c1));
  size_t n3 = 3 * (size_t)state_off;
  CK(c->xyz.alloc(n3)); CK(c->pxyz.alloc(n3)); CK(c->velo.alloc(n3)); CK(c->accel.alloc(n3));
  CK(c->dxyz.alloc(n3)); CK(c->out_force.alloc(n3)); CK(c->p0xyz.alloc(n3));
  CK(cudaMemset(c->p0xyz.p, 0, n3 * 8));
  CK(cudaMemset(c->xyz.p, 0, n3 * 8)); CK(cudaMemset(c->pxyz.p, 0, n3 * 8));
  CK(cudaMemset(c->velo.p, 0, n3 * 8)); CK(cudaMemset(c->accel.p, 0, n3 * 8));
  CK(cudaMemset(c->dxyz.p, 0, n3 * 8));
  CK(c->out_energy.alloc((size_t)nlane * N_ETYPE));
  CK(c->scale.alloc(nlane));
  CK(c->lane_n.alloc(nlane));
  CK(c->ebeta.alloc(nlane));
  CK(c->elabel.alloc(nlane));
  CK(c->e_opp.alloc((size_t)nlane * N_ETYPE));
  CK(c->rex_u.alloc((size_t)nlane / 2 + 1));
  CK(c->d_rep2lab.upload(c->rep2lab));
  CK(c->d_lab2rep.upload(c->lab2rep));
  {
    RexState r0{};
    r0.beta_global = c->beta_global;
    r0.counter = 0;
    r0.idx_pair = 1;
    r0.nacc = 0;
    CK(c->rex.upload(std::vector<RexState>{r0}));
  }
  CK(c->mask.alloc(mask_off));
  CK(cudaMemset(c->mask.p, 0, std::max<size_t>(mask_off, 1) * sizeof(uint32_t)));
  CK(c->mirror.alloc(periodic ? (size_t)mirror_off : 1));
  CK(c->slots.alloc(slot_off * 3 * real_size));
  CK(c->hb_flag.alloc(hb_off)); CK(c->hb_ene.alloc(hb_off)); CK(c->site_exc.alloc(site_off));
  CK(c->hb_flag2.alloc(hb_off)); CK(c->hb_ene2.alloc(hb_off)); CK(c->site_exc2.alloc(site_off));
  CK(cudaMemset(c->hb_flag.p, 0, std::max(hb_off, 1)));
  CK(cudaMemset(c->hb_ene.p, 0, std::max(hb_off, 1) * sizeof(double)));
  c->max_nmp = maxN;
  if (c->bdhi) {
    CK(c->fene_idx.upload(fene_idx)); CK(c->fene_nat.upload(fene_nat)); CK(c->fene_coef.upload(fene_coef));
    CK(c->fene_d2.upload(fene_d2));
    CK(c->wca_idx.upload(wca_idx)); CK(c->wca_nat.upload(wca_nat)); CK(c->wca_coef.upload(wca_coef));
    CK(c->bd_ptr.upload(bdp)); CK(c->bd_ent.upload(bde)); CK(c->b_hrad.upload(b_hrad));
    if (fene_cls.empty()) fene_cls.assign(3, 0.0);
    if (wca_cls.empty()) wca_cls.assign(3, 0.0);
    CK(c->fene_cls.upload(fene_cls)); CK(c->wca_cls.upload(wca_cls));
    if (p.precision == TIS_PREC_MIXED) {
      std::vector<int> lane_T, items;
      for (int l = 0; l < nlane; ++l) lane_T.push_back((3 * c->lane_nmp[l] + 63) / 64);
      if (*std::max_element(lane_T.begin(), lane_T.end()) > 500 || nlane > 32767) {
        tis_destroy(c);
        return TIS_E_UNSUPPORTED;   // work items pack the row block in 8 bits, the lane in 15
      }
      bd_update_items(lane_T, items, c->bd_koff);
      if (items.empty()) items.push_back(0);
      CK(c->bd_items.upload(items));
      CK(c->bd_D32.alloc((size_t)bd32_off)); CK(c->bd_L32.alloc((size_t)bd32_off));
      if (c->refine) {
        // z of a lane is staged in one CTA's shared memory
        if (3 * (size_t)maxN * 8 + 17 * 64 * 8 > 227 * 1024) { tis_destroy(c); return TIS_E_UNSUPPORTED; }
        CK(c->bd_D64.alloc((size_t)bd_off)); CK(c->bd_E32.alloc((size_t)bd32_off));
        CK(c->bd_W32.alloc((size_t)bdw_off)); CK(c->bd_z.alloc(n3));
        CK(cudaMemset(c->bd_E32.p, 0, (size_t)bd32_off * sizeof(float)));
      }
      // padding columns and the factor's upper part are never written
      CK(cudaMemset(c->bd_D32.p, 0, (size_t)bd32_off * sizeof(float)));
      CK(cudaMemset(c->bd_L32.p, 0, (size_t)bd32_off * sizeof(float)));
    } else {
      CK(c->bd_D.alloc((size_t)bd_off));
    }
    CK(c->bd_L.alloc((size_t)bd_off));
    CK(c->bd_W.alloc((size_t)nlane * 64 * 64));
    if (bdp_off) {
      CK(c->bd_P.alloc((size_t)bdp_off));
      CK(cudaMemset(c->bd_P.p, 0, (size_t)bdp_off * sizeof(float)));   // tile T of each lane stays zero
    }
    CK(c->bd_F.alloc(n3)); CK(c->bd_xi.alloc(n3));
    CK(cudaMemset(c->bd_F.p, 0, n3 * 8));
    CK(c->d_not_spd.alloc(nlane));
    CK(cudaMemset(c->d_not_spd.p, 0, nlane * sizeof(int)));
  }
  if (p.i_ele == TIS_ELE_EWALD) {
    std::vector<int8_t> h;
    std::vector<double> coef;
    ewald_table(p.psize[0], p.ewld_alpha, p.ewld_hmax, h, coef);
    c->nk = (int)coef.size();
    c->hmax = (int)std::ceil(p.ewld_hmax);
    c->nqblk = std::min(16, std::max(1, (c->nq_max + 63) / 64));
    CK(c->ew_h.upload(h));
    CK(c->ew_coef.upload(coef));
    CK(c->ew_tab.alloc(std::max<size_t>((size_t)ew_off * 3 * (c->hmax + 1) * 2, 1)));
    CK(c->ew_S.alloc(std::max<size_t>((size_t)nlane * c->nqblk * c->nk * 2, 1)));
    CK(c->f_ext.alloc(n3 * EW_F_SPLIT));
    CK(cudaMemset(c->f_ext.p, 0, n3 * EW_F_SPLIT * 8));
  }
  c->clamp_seen.assign(nlane, 0);
  *out = c;
  return TIS_OK;
}
}  // namespace

extern "C" int tis_init_batch(int32_t ntop, const tis_topology *tops, const tis_params *par,
                              const int32_t *nrep, const double *tempk, tis_ctx **out) {
  return init_impl(ntop, tops, par, nrep, tempk, nullptr, out);
}

extern "C" int tis_init_ladder(const tis_topology *top, const tis_params *par, int32_t nrep_all,
                               const double *tempk_all, int32_t irep_first, int32_t nrep_local, tis_ctx **out) {
  if (!out || !tempk_all || nrep_all <= 0 || nrep_local <= 0 || irep_first < 1 ||
      irep_first - 1 + nrep_local > nrep_all)
    return TIS_E_ARG;
  if (par && par->i_simulate_type == TIS_SIM_BROWNIAN_HI) return TIS_E_UNSUPPORTED;
  const Ladder lad{nrep_all, tempk_all, irep_first - 1};
  return init_impl(1, top, par, &nrep_local, nullptr, &lad, out);
}

extern "C" int tis_init(const tis_topology *top, const tis_params *par, int32_t nrep, const double *tempk,
                        tis_ctx **out) {
  if (nrep <= 0) return TIS_E_ARG;
  return tis_init_batch(1, top, par, &nrep, tempk, out);
}

extern "C" void tis_destroy(tis_ctx *c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  c->d_tops.free(); c->d_lanes.free(); c->d_lstate.free();
  c->b_type.free(); c->b_class.free(); c->b_unit.free();
  c->b_rcmass.free(); c->b_cmass.free(); c->b_fric.free(); c->b_radius.free(); c->b_eps.free(); c->b_charge.free();
  c->b_c2.free(); c->b_c3.free(); c->b_c4.free(); c->b_screen.free();
  c->u_lunit.free(); c->u_class.free(); c->rneigh2.free();
  c->bd_idx.free(); c->ba_idx.free(); c->st_idx.free(); c->hb_idx.free(); c->hb_site.free();
  c->tst_idx.free(); c->tst_nat.free(); c->tst_coef.free(); c->stx_ptr.free(); c->stx_tst.free();
  c->site_val.free(); c->site_ptr.free(); c->site_hb.free(); c->inc_ptr.free(); c->inc_slot.free();
  c->q_bead.free();
  c->bd_nat.free(); c->bd_coef.free(); c->ba_nat.free(); c->ba_coef.free(); c->st_nat.free(); c->st_coef.free();
  c->hb_nat.free(); c->hb_coef.free(); c->hb_nd2.free(); c->hb_tert.free(); c->b_qkind.free(); c->lab_zp.free(); c->pmf_e.free(); c->pmf_f.free();
  c->lab_Td.free(); c->lab_coef.free(); c->lab_cdist.free(); c->lab_beta.free(); c->lab_rele2.free();
  c->lab_u0.free(); c->lab_c1.free(); c->lab_u0off.free(); c->lab_c1off.free(); c->elabel.free();
  c->ebeta.free(); c->e_opp.free(); c->rex_u.free(); c->d_rep2lab.free(); c->d_lab2rep.free(); c->rex.free();
  c->xyz.free(); c->pxyz.free(); c->velo.free(); c->accel.free(); c->dxyz.free(); c->p0xyz.free();
  c->out_force.free(); c->out_energy.free(); c->scale.free();
  c->mask.free(); c->site_exc.free(); c->mirror.free(); c->hb_flag.free();
  c->hb_ene.free(); c->hb_flag2.free(); c->hb_ene2.free(); c->site_exc2.free(); c->slots.free(); c->noise.free(); c->unif.free(); c->lane_n.free(); c->d_order.free();
  c->ew_h.free(); c->ew_coef.free(); c->ew_tab.free(); c->ew_S.free(); c->f_ext.free();
  c->fene_idx.free(); c->wca_idx.free(); c->bd_ptr.free(); c->bd_ent.free(); c->fene_cls.free(); c->wca_cls.free(); c->b_hrad.free(); c->d_not_spd.free();
  c->fene_nat.free(); c->fene_coef.free(); c->fene_d2.free(); c->wca_nat.free(); c->wca_coef.free();
  c->bd_D64.free(); c->bd_z.free(); c->bd_E32.free(); c->bd_W32.free();
  c->bd_D.free(); c->bd_L.free(); c->bd_P.free(); c->bd_items.free(); c->bd_D32.free(); c->bd_L32.free(); c->bd_W.free(); c->bd_F.free(); c->bd_xi.free();
  if (c->g_exec) cudaGraphExecDestroy(c->g_exec);
  if (c->g_ev0) cudaEventDestroy(c->g_ev0);
  if (c->g_ev1) cudaEventDestroy(c->g_ev1);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->tev0) cudaEventDestroy(c->tev0);
  if (c->tev1) cudaEventDestroy(c->tev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" int tis_nrep(const tis_ctx *c) { return c ? c->nlane : TIS_E_ARG; }
extern "C" int tis_nmp(const tis_ctx *c, int32_t irep) {
  if (!c || irep < 1 || irep > c->nlane) return TIS_E_ARG;
  return c->lane_nmp[irep - 1];
}

// ------------------------------------------------------------------- state
extern "C" int tis_set_state(tis_ctx *c, const double *xyz, const double *velo, const double *accel) {
  if (!c || !xyz) return TIS_E_ARG;
  size_t n = 3 * (size_t)c->nbead_total * sizeof(double);
  CK(cudaMemcpyAsync(c->xyz.p, xyz, n, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->pxyz.p, xyz, n, cudaMemcpyHostToDevice, c->stream));
  if (velo) CK(cudaMemcpyAsync(c->velo.p, velo, n, cudaMemcpyHostToDevice, c->stream));
  else CK(cudaMemsetAsync(c->velo.p, 0, n, c->stream));
  if (accel) CK(cudaMemcpyAsync(c->accel.p, accel, n, cudaMemcpyHostToDevice, c->stream));
  else CK(cudaMemsetAsync(c->accel.p, 0, n, c->stream));
  CK(cudaMemsetAsync(c->dxyz.p, 0, n, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return TIS_OK;
}

extern "C" int tis_get_state(tis_ctx *c, double *xyz, double *velo, double *accel) {
  if (!c) return TIS_E_ARG;
  size_t n = 3 * (size_t)c->nbead_total * sizeof(double);
  if (xyz) CK(cudaMemcpyAsync(xyz, c->xyz.p, n, cudaMemcpyDeviceToHost, c->stream));
  if (velo) CK(cudaMemcpyAsync(velo, c->velo.p, n, cudaMemcpyDeviceToHost, c->stream));
  if (accel) CK(cudaMemcpyAsync(accel, c->accel.p, n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return TIS_OK;
}

namespace {
KArgs make_args(tis_ctx *c, int mode, int nsteps, int only_lane);
}  // namespace

extern "C" int tis_set_step(tis_ctx *c, int64_t istep) {
  if (!c || istep < 0) return TIS_E_ARG;
  std::vector<LaneState> ls(c->nlane);
  CK(cudaMemcpyAsync(ls.data(), c->d_lstate.p, ls.size() * sizeof(LaneState), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (auto &l : ls) l.istep = istep;
  CK(cudaMemcpyAsync(c->d_lstate.p, ls.data(), ls.size() * sizeof(LaneState), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->bd_istep = istep;
  return TIS_OK;
}

extern "C" int tis_get_dtrna_status(tis_ctx *c, int32_t irep, int32_t *hb_status, int32_t *st_status) {
  if (!c || irep < 1 || irep > c->nlane) return TIS_E_ARG;
  const LaneDesc &L = c->lanes[irep - 1];
  const TopDesc &T = c->tops[L.top];
  if (hb_status && T.nhb > 0) {
    std::vector<uint8_t> f(T.nhb);
    CK(cudaMemcpyAsync(f.data(), c->hb_flag.p + L.hb0, T.nhb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int h = 0; h < T.nhb; ++h) hb_status[h] = (f[h] & 2) ? 1 : 0;
  }
  if (st_status && T.nst > 0) {
    DBuf<int> out;
    CK(out.alloc(T.nst));
    KArgs a = make_args(c, 0, 0, irep - 1);
    ++c->launches;
    CK(st_status_launch(c->stream, a, irep - 1, T.nst, out.p));
    CK(cudaMemcpyAsync(st_status, out.p, T.nst * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    out.free();
  }
  return TIS_OK;
}

extern "C" int tis_get_pxyz(tis_ctx *c, double *pxyz) {
  if (!c || !pxyz) return TIS_E_ARG;
  CK(cudaMemcpy(pxyz, c->pxyz.p, 3 * (size_t)c->nbead_total * sizeof(double), cudaMemcpyDeviceToHost));
  return TIS_OK;
}

extern "C" int tis_set_noise(tis_ctx *c, const double *noise, int32_t nsteps, const double *uniforms, int32_t n_uniform) {
  if (!c) return TIS_E_ARG;
  if (noise && nsteps > 0) {
    std::vector<double> tmp(noise, noise + 3 * (size_t)c->nbead_total * nsteps);
    CK(c->noise.upload(tmp));
    c->noise_nsteps = nsteps;
  } else {
    c->noise.free();
    c->noise_nsteps = 0;
  }
  c->noise_base = 0;
  if (uniforms && n_uniform > 0) {
    std::vector<double> tmp(uniforms, uniforms + (size_t)n_uniform * c->nlane);
    CK(c->unif.upload(tmp));
    c->n_unif = n_uniform;
    for (int i = 0; i < c->nlane; ++i) c->lanes[i].unif0 = i * n_uniform;
  } else {
    c->unif.free();
    c->n_unif = 0;
    for (int i = 0; i < c->nlane; ++i) c->lanes[i].unif0 = 0;
  }
  CK(cudaMemcpy(c->d_lanes.p, c->lanes.data(), c->lanes.size() * sizeof(LaneDesc), cudaMemcpyHostToDevice));
  // reset the per-lane uniform positions
  std::vector<LaneState> ls(c->nlane);
  CK(cudaMemcpy(ls.data(), c->d_lstate.p, ls.size() * sizeof(LaneState), cudaMemcpyDeviceToHost));
  for (auto &s : ls) { s.unif_pos = 0; s.flags &= ~(LF_UNIF_EXHAUSTED | LF_NOISE_EXHAUSTED); }
  CK(cudaMemcpy(c->d_lstate.p, ls.data(), ls.size() * sizeof(LaneState), cudaMemcpyHostToDevice));
  return TIS_OK;
}

// -------------------------------------------------------------- launches
namespace {

KArgs make_args(tis_ctx *c, int mode, int nsteps, int only_lane) {
  const tis_params &p = c->par;
  KArgs a{};
  a.nlane = c->nlane;
  a.nsteps = nsteps;
  a.mode = mode;
  a.only_lane = only_lane;
  a.group = c->group;
  a.periodic = p.i_periodic == 1;
  for (int d = 0; d < 3; ++d) { a.psize[d] = p.psize[d]; a.psizeh[d] = p.psize[d] / 2.0; }
  a.neigh_margin = p.neigh_margin;
  a.n_step_neighbor = p.n_step_neighbor;
  a.exv_dist = p.exv_dist; a.exv_dist_PS = p.exv_dist_PS; a.exv_adjust = p.exv_adjust; a.exv_inf = p.exv_inf;
  a.nsep[0] = p.n_sep_nlocal_P; a.nsep[1] = p.n_sep_nlocal_S; a.nsep[2] = p.n_sep_nlocal_B;
  a.i_ele = (p.i_ele == TIS_ELE_DH) ? 1 : (p.i_ele == TIS_ELE_EWALD ? 2 : (p.i_ele == TIS_ELE_COULOMB ? 3 : 0));
  if (p.i_ele == TIS_ELE_EWALD) {
    a.ewld_alpha = p.ewld_alpha;
    a.ewld_beta = 2.0 * p.ewld_alpha / std::sqrt(F_PI);
    a.ewld_self = -p.ewld_alpha / std::sqrt(F_PI);
    a.nk = c->nk; a.hmax = c->hmax; a.nqblk = c->nqblk;
    for (int d = 0; d < 3; ++d) a.two_pi_L[d] = 2.0 * F_PI / p.psize[0];
    a.ew_h = c->ew_h.p; a.ew_coef = c->ew_coef.p; a.ew_tab = c->ew_tab.p; a.ew_S = c->ew_S.p;
  }
  a.f_ext = nullptr;
  a.fene_idx = c->fene_idx.p; a.fene_nat = c->fene_nat.p; a.fene_coef = c->fene_coef.p; a.fene_d2 = c->fene_d2.p;
  a.wca_idx = c->wca_idx.p; a.wca_nat = c->wca_nat.p; a.wca_coef = c->wca_coef.p;
  a.wca_rcut2 = 1.0 / (p.wca_coef_cutoff * p.wca_coef_cutoff);
  a.bd_ptr = c->bd_ptr.p; a.bd_ent = c->bd_ent.p; a.fene_cls = c->fene_cls.p; a.wca_cls = c->wca_cls.p;
  a.bd_D = c->bd_D.p; a.bd_L = c->bd_L.p; a.bd_P = c->bd_P.p; a.bd_D32 = c->bd_D32.p; a.bd_L32 = c->bd_L32.p; a.bd_W = c->bd_W.p; a.bd_F = c->bd_F.p; a.bd_xi = c->bd_xi.p;
  a.not_spd = c->d_not_spd.p;
  a.bd_refine = c->refine ? 1 : 0;
  a.bd_D64 = c->bd_D64.p; a.bd_E32 = c->bd_E32.p; a.bd_W32 = c->bd_W32.p; a.bd_z = c->bd_z.p;
  a.hi_radius = p.hi_radius; a.viscosity = p.viscosity;
  a.i_hydro_tensor = p.i_hydro_tensor == 0 ? TIS_HI_RPY : p.i_hydro_tensor;
  a.b_hrad = c->b_hrad.p;
  a.boltz = BOLTZ_KCAL_MOL; a.pi = F_PI;
  a.bd_istep = c->bd_istep; a.bd_kpanel = 0;
  a.bd_tc = (c->bdhi && p.precision == TIS_PREC_MIXED) ? 1 : 0;
  a.cutoff_ele = p.cutoff_ele;
  a.i_DH_cutoff_type = p.i_DH_cutoff_type;
  a.hb_cutoff_dist = p.hb_cutoff_dist;
  a.max_abscos = std::cos((double)(0.57f / 180.0f) * F_PI);
  a.tstep = p.tstep; a.tstep2 = 0.5e0 * p.tstep * p.tstep; a.tsteph = 0.5e0 * p.tstep;
  a.beta_hbond15 = c->beta_global;
  a.rex = c->rex.p;
  a.hb_beta_global = p.hb_beta_global;
  a.seed = p.seed;
  a.tops = c->d_tops.p; a.lanes = c->d_lanes.p; a.lstate = c->d_lstate.p;
  a.b_type = c->b_type.p; a.b_class = c->b_class.p; a.b_unit = c->b_unit.p;
  a.b_rcmass = c->b_rcmass.p; a.b_cmass = c->b_cmass.p; a.b_fric = c->b_fric.p; a.b_radius = c->b_radius.p;
  a.b_eps = c->b_eps.p; a.b_charge = c->b_charge.p; a.b_screen = c->b_screen.p;
  a.u_lunit = c->u_lunit.p; a.u_class = c->u_class.p; a.rneigh2 = c->rneigh2.p;
  a.bd_idx = c->bd_idx.p; a.bd_nat = c->bd_nat.p; a.bd_coef = c->bd_coef.p;
  a.ba_idx = c->ba_idx.p; a.ba_nat = c->ba_nat.p; a.ba_coef = c->ba_coef.p;
  a.st_idx = c->st_idx.p; a.st_nat = c->st_nat.p; a.st_coef = c->st_coef.p;
  a.tst_idx = c->tst_idx.p; a.tst_nat = c->tst_nat.p; a.tst_coef = c->tst_coef.p;
  a.stx_ptr = c->stx_ptr.p; a.stx_tst = c->stx_tst.p;
  a.hb_idx = c->hb_idx.p; a.hb_nat = c->hb_nat.p; a.hb_coef = c->hb_coef.p; a.hb_site = c->hb_site.p;
  a.hb_tert = c->hb_tert.p;
  a.dt19 = p.i_dtrna_model == 2019;
  a.b_qkind = c->b_qkind.p; a.lab_zp = c->lab_zp.p;
  a.pmf_e = c->pmf_e.p; a.pmf_f = c->pmf_f.p;
  a.pmf_nbin = p.pmf_nbin; a.pmf_rmin = p.pmf_rmin; a.pmf_rbin = p.pmf_rbin; a.pmf_rmax = p.pmf_rmax;
  a.pmf_rbininv = (p.pmf_rbin > 0.0) ? 1.0 / p.pmf_rbin : 0.0;
  a.hb_nd2 = c->hb_nd2.p;
  a.site_val = c->site_val.p; a.site_ptr = c->site_ptr.p; a.site_hb = c->site_hb.p;
  a.inc_ptr = c->inc_ptr.p; a.inc_slot = c->inc_slot.p; a.q_bead = c->q_bead.p;
  a.lab_T = c->lab_Td.p; a.lab_coef = c->lab_coef.p; a.lab_cdist = c->lab_cdist.p; a.lab_beta = c->lab_beta.p;
  a.lab_rele2 = c->lab_rele2.p; a.lab_u0off = c->lab_u0off.p; a.lab_u0 = c->lab_u0.p;
  a.lab_c1off = c->lab_c1off.p; a.lab_c1 = c->lab_c1.p;
  a.b_c2 = c->b_c2.p; a.b_c3 = c->b_c3.p; a.b_c4 = c->b_c4.p;
  a.xyz = c->xyz.p; a.pxyz = c->pxyz.p; a.velo = c->velo.p; a.accel = c->accel.p; a.dxyz = c->dxyz.p;
  a.p0xyz = c->p0xyz.p;
  a.mask = c->mask.p; a.mirror = c->mirror.p;
  a.smem_total = (int)c->smem;
  a.slots = c->slots.p; a.hb_flag = c->hb_flag.p; a.hb_ene = c->hb_ene.p; a.site_exc = c->site_exc.p;
  a.elabel = nullptr; a.reuse_hb = 0; a.ebeta = c->beta_global; a.out_energy = c->out_energy.p;
  a.out_force = c->out_force.p;
  a.noise = c->noise_nsteps ? c->noise.p : nullptr;
  a.noise_nsteps = c->noise_nsteps;
  a.noise_base = c->noise_base;
  a.unif = c->n_unif ? c->unif.p : nullptr;
  a.n_unif = c->n_unif;
  a.nbead_total = c->nbead_total;
  a.noise_in_sweep = 0;
  a.sweep_mode = c->sweep - 1;
  a.lane_nsteps = nullptr;
  a.step_k = 0;
  a.lane_order = (c->order == 2 && only_lane < 0) ? c->d_order.p : nullptr;
  return a;
}

// Ewald reciprocal space for the lanes of `a` (tables, structure factors
// and, when `forces`, the per-charge forces in f_ext, which the next lane
// launch adds to each bead's sum).  No-op without Ewald.
int ewald_recip(tis_ctx *c, KArgs &a, bool forces) {
  if (c->par.i_ele != TIS_ELE_EWALD) return TIS_OK;
  c->launches += (forces ? 3 : 2) + (c->nqblk > 1 ? 1 : 0);
  if (forces) a.f_ext = c->f_ext.p;   // written by the force kernel, read by the lane kernel
  CK(ewald_recip_launch(c->stream, a, c->nq_max, forces));
  return TIS_OK;
}

int launch_lane(tis_ctx *c, const KArgs &a) {
  ++c->launches;
  CK(lane_kernel_launch(c->par.precision == TIS_PREC_MIXED, a.only_lane >= 0 ? 1 : a.nlane, c->threads, c->smem,
                        c->stream, a));
  return TIS_OK;
}

int check_lanes(tis_ctx *c) {
  std::vector<LaneState> ls(c->nlane);
  CK(cudaMemcpyAsync(ls.data(), c->d_lstate.p, ls.size() * sizeof(LaneState), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  long long clamps = 0;
  int code = TIS_OK;
  for (int i = 0; i < c->nlane; ++i) {
    if (ls[i].flags & LF_NAN) code = fail(c, TIS_E_NAN, "non-finite force in lane " + std::to_string(i + 1));
    if (ls[i].flags & LF_PMF)
      code = fail(c, TIS_E_PMF_RANGE, "Mg-P pair below the PMF table in lane " + std::to_string(i + 1));
    if (ls[i].flags & LF_OVERFLOW) code = fail(c, TIS_E_LIST_OVERFLOW, "hbond site list overflow");
    if (ls[i].flags & LF_SMEM)
      code = fail(c, TIS_E_UNSUPPORTED, "the shared-memory layout of lane " + std::to_string(i + 1) + " does not fit");
    if (ls[i].flags & (LF_UNIF_EXHAUSTED | LF_NOISE_EXHAUSTED))
      code = fail(c, TIS_E_NOISE_EXHAUSTED, "injected noise or uniforms exhausted");
    clamps += ls[i].nclamp - c->clamp_seen[i];
    c->clamp_seen[i] = ls[i].nclamp;
  }
  if (c->bdhi) {
    std::vector<int> ns(c->nlane);
    CK(cudaMemcpy(ns.data(), c->d_not_spd.p, ns.size() * sizeof(int), cudaMemcpyDeviceToHost));
    for (int i = 0; i < c->nlane; ++i) {
      if (ns[i] & 1) {
        c->not_spd = 1;
        code = fail(c, TIS_E_NOT_SPD, "Cholesky factorisation of the diffusion tensor failed in lane " +
                                          std::to_string(i + 1));
      }
      if (ns[i] & 2) {
        c->wait_timeout = 1;
        code = fail(c, TIS_E_TIMEOUT, "tensor-core update of the Cholesky factor did not complete");
      }
    }
  }
  if (code < 0) return code;
  return (int)std::min<long long>(clamps, 0x7fffffff);
}

}  // namespace

extern "C" int tis_neighbor(tis_ctx *c, int32_t irep) {
  if (!c || irep == 0 || irep > c->nlane || irep < -1) return TIS_E_ARG;
  if (c->bdhi) return TIS_OK;   // no pair-list terms on the Brownian-HI path
  KArgs a = make_args(c, KM_NEIGHBOR, 0, irep > 0 ? irep - 1 : -1);
  int rc = launch_lane(c, a);
  if (rc < 0) return rc;
  return check_lanes(c);
}

namespace {
// Copies the lane's list bit matrices (and mirror indices) back.
int fetch_masks(tis_ctx *c, int lane, std::vector<uint32_t> &m, std::vector<uint8_t> &mir) {
  const LaneDesc &L = c->lanes[lane];
  const int N = c->lane_nmp[lane], W = (N + 31) / 32;
  m.resize(2 * (size_t)N * W);
  CK(cudaMemcpy(m.data(), c->mask.p + L.mask0, m.size() * 4, cudaMemcpyDeviceToHost));
  if (c->par.i_periodic == 1) {
    mir.resize((size_t)N * N);
    CK(cudaMemcpy(mir.data(), c->mirror.p + L.mirror0, mir.size(), cudaMemcpyDeviceToHost));
  }
  return TIS_OK;
}
}  // namespace

extern "C" int tis_get_exv_list(tis_ctx *c, int32_t irep, int32_t *iexv2mp, int32_t cap, int32_t *n) {
  if (!c || irep < 1 || irep > c->nlane) return TIS_E_ARG;
  std::vector<uint32_t> m;
  std::vector<uint8_t> mir;
  int rc = fetch_masks(c, irep - 1, m, mir);
  if (rc < 0) return rc;
  const int N = c->lane_nmp[irep - 1], W = (N + 31) / 32;
  const bool peri = c->par.i_periodic == 1;
  int k = 0;
  for (int i = 0; i < N; ++i)
    for (int j = i + 1; j < N; ++j) {
      if (!(m[(size_t)i * W + (j >> 5)] >> (j & 31) & 1u)) continue;
      if (k < cap && iexv2mp) {
        iexv2mp[3 * k] = i + 1;
        iexv2mp[3 * k + 1] = j + 1;
        iexv2mp[3 * k + 2] = peri ? (int)mir[(size_t)i * N + j] : 1;
      }
      ++k;
    }
  if (n) *n = k;
  return k > cap ? TIS_E_LIST_OVERFLOW : TIS_OK;
}

extern "C" int tis_get_ele_list(tis_ctx *c, int32_t irep, int32_t *iele2mp, double *coef_ele, int32_t cap, int32_t *n) {
  if (!c || irep < 1 || irep > c->nlane) return TIS_E_ARG;
  std::vector<uint32_t> m;
  std::vector<uint8_t> mir;
  const int lane = irep - 1;
  int rc = fetch_masks(c, lane, m, mir);
  if (rc < 0) return rc;
  const TopDesc &T = c->tops[c->lanes[lane].top];
  const int N = T.nmp, W = (N + 31) / 32;
  const bool peri = c->par.i_periodic == 1;
  const uint32_t *mele = m.data() + (size_t)N * W;
  std::vector<double> q(N);
  std::vector<int8_t> typ(N);
  CK(cudaMemcpy(q.data(), c->b_charge.p + T.bead0, N * sizeof(double), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(typ.data(), c->b_type.p + T.bead0, N, cudaMemcpyDeviceToHost));
  std::vector<LaneState> ls(1);
  CK(cudaMemcpy(ls.data(), c->d_lstate.p + lane, sizeof(LaneState), cudaMemcpyDeviceToHost));
  double coefT = 0.0;
  CK(cudaMemcpy(&coefT, c->lab_coef.p + ls[0].label, sizeof(double), cudaMemcpyDeviceToHost));
  if (c->b_qkind.p) {   // i_charge = 1: the label's phosphate charge
    std::vector<uint8_t> qk(N);
    double zp = 0.0;
    CK(cudaMemcpy(qk.data(), c->b_qkind.p + T.bead0, N, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&zp, c->lab_zp.p + ls[0].label, sizeof(double), cudaMemcpyDeviceToHost));
    for (int i = 0; i < N; ++i)
      if (qk[i]) q[i] = -zp;
  }
  const bool dt19 = c->par.i_dtrna_model == 2019;
  int k = 0;
  for (int i = 0; i < N; ++i)
    for (int j = i + 1; j < N; ++j) {
      if (!(mele[(size_t)i * W + (j >> 5)] >> (j & 31) & 1u)) continue;
      if (k < cap) {
        if (iele2mp) {
          iele2mp[4 * k] = i + 1;
          iele2mp[4 * k + 1] = j + 1;
          iele2mp[4 * k + 2] = peri ? (int)mir[(size_t)i * N + j] : 1;
          // neighbor_list_ele.F90:167-174: PMFTYPE%MG_P = 1 for Mg-P pairs of the DT19 model
          iele2mp[4 * k + 3] = (dt19 && ((typ[i] == TIS_MP_RNA_PHOS && typ[j] == TIS_MP_ION_MG) ||
                                         (typ[i] == TIS_MP_ION_MG && typ[j] == TIS_MP_RNA_PHOS))) ? 1 : 0;
        }
        if (coef_ele) coef_ele[k] = q[i] * q[j] * coefT;
      }
      ++k;
    }
  if (n) *n = k;
  return k > cap ? TIS_E_LIST_OVERFLOW : TIS_OK;
}

extern "C" int tis_get_hb_list(tis_ctx *c, int32_t irep, int32_t *ineigh2hb, int32_t cap, int32_t *n) {
  if (!c || irep < 1 || irep > c->nlane) return TIS_E_ARG;
  const LaneDesc &L = c->lanes[irep - 1];
  const TopDesc &T = c->tops[L.top];
  std::vector<uint8_t> f(std::max(T.nhb, 1));
  if (T.nhb) CK(cudaMemcpy(f.data(), c->hb_flag.p + L.hb0, T.nhb, cudaMemcpyDeviceToHost));
  int k = 0;
  for (int h = 0; h < T.nhb; ++h)
    if (f[h] & 1) {
      if (k < cap && ineigh2hb) ineigh2hb[k] = h + 1;
      ++k;
    }
  if (n) *n = k;
  return k > cap ? TIS_E_LIST_OVERFLOW : TIS_OK;
}

extern "C" int tis_force_sumup(tis_ctx *c, int32_t irep, double *force_mp) {
  if (!c || irep < 1 || irep > c->nlane) return TIS_E_ARG;
  if (c->bdhi) {
    KArgs a = make_args(c, 0, 0, -1);
    ++c->launches;
    CK(bd_force_launch(c->stream, a, c->max_nmp));
    const LaneDesc &L = c->lanes[irep - 1];
    if (force_mp)
      CK(cudaMemcpyAsync(force_mp, c->bd_F.p + 3 * (size_t)L.state0, 3 * (size_t)c->lane_nmp[irep - 1] * 8,
                         cudaMemcpyDeviceToHost, c->stream));
    return check_lanes(c);
  }
  KArgs a = make_args(c, KM_FORCE, 0, irep - 1);
  int rc = ewald_recip(c, a, true);
  if (rc < 0) return rc;
  rc = launch_lane(c, a);
  if (rc < 0) return rc;
  c->hb_energy_valid = true;
  const LaneDesc &L = c->lanes[irep - 1];
  if (force_mp)
    CK(cudaMemcpyAsync(force_mp, c->out_force.p + 3 * (size_t)L.state0, 3 * (size_t)c->lane_nmp[irep - 1] * 8,
                       cudaMemcpyDeviceToHost, c->stream));
  return check_lanes(c);
}

namespace {
int run_energy(tis_ctx *c, int only_lane, const int *labels, bool reuse, double beta, std::vector<double> &E,
               const double *beta_lane = nullptr) {
  KArgs a = make_args(c, 0, 0, only_lane);
  if (labels) {
    CK(cudaMemcpyAsync(c->elabel.p, labels, c->nlane * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    a.elabel = c->elabel.p;
  }
  if (beta_lane) {
    CK(cudaMemcpyAsync(c->ebeta.p, beta_lane, c->nlane * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    a.ebeta_lane = c->ebeta.p;
  }
  a.reuse_hb = reuse ? 1 : 0;
  a.ebeta = beta;
  ++c->launches;
  CK(energy_kernel_launch(only_lane >= 0 ? 1 : c->nlane, c->max_nmp, c->stream, a));
  if (c->par.i_ele == TIS_ELE_EWALD) {
    int rc = ewald_recip(c, a, false);
    if (rc < 0) return rc;
    ++c->launches;
    CK(ewald_energy_launch(c->stream, a));
  }
  E.resize((size_t)c->nlane * N_ETYPE);
  CK(cudaMemcpyAsync(E.data(), c->out_energy.p, E.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return TIS_OK;
}
}  // namespace

extern "C" int tis_energy_sumup(tis_ctx *c, int32_t irep, double *energy) {
  if (!c || irep < 1 || irep > c->nlane || !energy) return TIS_E_ARG;
  std::vector<double> E;
  int rc = run_energy(c, irep - 1, nullptr, c->hb_energy_valid, c->beta_global, E);
  if (rc < 0) return rc;
  std::memcpy(energy, &E[(size_t)(irep - 1) * N_ETYPE], N_ETYPE * sizeof(double));
  return check_lanes(c);
}

extern "C" int tis_time_integral_pre(tis_ctx *c) {
  if (!c) return TIS_E_ARG;
  if (c->bdhi) {
    // time_integral_pre.F90:313-317: velocities zero; forces at x0
    const size_t n3 = 3 * (size_t)c->nbead_total;
    CK(cudaMemsetAsync(c->velo.p, 0, n3 * 8, c->stream));
    CK(cudaMemsetAsync(c->accel.p, 0, n3 * 8, c->stream));
    CK(cudaMemsetAsync(c->dxyz.p, 0, n3 * 8, c->stream));
    KArgs a = make_args(c, 0, 0, -1);
    ++c->launches;
    CK(bd_force_launch(c->stream, a, c->max_nmp));
    c->noise_base += 1;
    return check_lanes(c);
  }
  KArgs a = make_args(c, KM_PRE, 0, -1);
  int rc = ewald_recip(c, a, true);
  if (rc < 0) return rc;
  rc = launch_lane(c, a);
  if (rc < 0) return rc;
  c->noise_base += 1;
  c->hb_energy_valid = true;
  return check_lanes(c);
}

namespace {
// The kernels of nsteps steps of every lane, queued on the context's stream
// without a host wait (lane_n_dev: per-lane step counts on the device, or
// NULL).  Outside the Brownian-HI path (whose refresh schedule is counted
// on the host) every launch argument is fixed when it is queued, so the
// same sequence can be recorded into a CUDA graph (tis_run).
int enqueue_steps(tis_ctx *c, int nsteps, const int *lane_n_dev) {
  KArgs a = make_args(c, KM_STEP, nsteps, -1);
  a.lane_nsteps = lane_n_dev;
  if (c->pair) {
    a.smem_total = (int)c->smem2;
    // the two-CTA sweep has idle warps: the sink's noise is drawn there
    a.noise_in_sweep = c->noise_sweep == 1 ? 1 : 0;
    ++c->launches;
    CK(lane_kernel_launch_pair(c->nlane, c->smem2, c->stream, a));
  } else if (c->bdhi) {
    // time_integral.F90:429-457, all lanes together
    const int every = c->par.n_step_hydro > 0 ? c->par.n_step_hydro : 1;
    for (int64_t k = 0; k < nsteps; ++k) {
      const long long istep = c->bd_istep + 1;
      KArgs b = make_args(c, 0, 0, -1);
      b.bd_istep = istep;
      b.noise_base = c->noise_base + (int)k;
      if ((istep - 1) % every == 0) {
        c->launches += bd_refactor_launches(c->max_nmp, b.bd_tc != 0) + (c->refine ? 2 : 0);
        CK(bd_refactor_launch(c->stream, b, c->max_nmp, c->bd_items.p, c->bd_koff.data()));
      }
      c->launches += 3 + (c->refine ? 1 : 0);
      CK(bd_step_launch(c->stream, b, c->max_nmp));
      c->bd_istep = istep;
    }
  } else if (c->par.i_ele != TIS_ELE_EWALD) {
    int rc = launch_lane(c, a);
    if (rc < 0) return rc;
  } else {
    // the reciprocal sum needs every charge's new position: each step is
    // x update -> reciprocal forces -> forces, v / a update; the x update
    // of step k + 1 runs in the launch of step k's forces
    KArgs x = make_args(c, KM_XSTEP, 1, -1);
    x.lane_nsteps = a.lane_nsteps;
    x.step_k = 0;
    int rc = launch_lane(c, x);
    if (rc < 0) return rc;
    for (int64_t k = 0; k < nsteps; ++k) {
      KArgs v = make_args(c, k + 1 < nsteps ? KM_VXSTEP : KM_VSTEP, 1, -1);
      v.lane_nsteps = a.lane_nsteps;
      v.step_k = (int)k;
      v.noise_base = c->noise_base + (int)k;
      rc = ewald_recip(c, v, true);
      if (rc < 0) return rc;
      rc = launch_lane(c, v);
      if (rc < 0) return rc;
    }
  }
  return TIS_OK;
}

// nsteps calls of time_integral for every lane; lane_n (host, per lane, may
// be null) lets lane l take only lane_n[l] of them (replicas that wait for
// their exchange step, time_integral.F90:134).
int run_steps(tis_ctx *c, int nsteps, const std::vector<int> *lane_n) {
  const int *lane_n_dev = nullptr;
  if (lane_n) {
    if (c->bdhi) return fail(c, TIS_E_UNSUPPORTED, "per-replica step counts on the Brownian-HI path");
    CK(cudaMemcpyAsync(c->lane_n.p, lane_n->data(), c->nlane * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    lane_n_dev = c->lane_n.p;
  }
  CK(cudaEventRecord(c->ev0, c->stream));
  const int rc = enqueue_steps(c, nsteps, lane_n_dev);
  if (rc < 0) return rc;
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  c->noise_base += (int)nsteps;
  c->hb_energy_valid = true;
  return check_lanes(c);
}
}  // namespace

extern "C" int tis_step(tis_ctx *c, int64_t nsteps) {
  if (!c || nsteps < 0 || nsteps > 0x7fffffff) return TIS_E_ARG;
  if (nsteps == 0) return TIS_OK;
  return run_steps(c, (int)nsteps, nullptr);
}

extern "C" int tis_time_integral(tis_ctx *c, int64_t nsteps, int32_t *flg, const int64_t *exchange_step) {
  if (!c || !flg || nsteps < 0 || nsteps > 0x7fffffff) return TIS_E_ARG;
  if (nsteps == 0) return TIS_OK;
  std::vector<LaneState> ls(c->nlane);
  CK(cudaMemcpyAsync(ls.data(), c->d_lstate.p, ls.size() * sizeof(LaneState), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::vector<int> n(c->nlane);
  for (int l = 0; l < c->nlane; ++l) {
    long long k = flg[l] ? 0 : nsteps;
    if (!flg[l] && exchange_step) {
      const long long left = exchange_step[l] - ls[l].istep;
      k = std::max(0LL, std::min(k, left));
    }
    n[l] = (int)k;
  }
  const int rc = run_steps(c, (int)nsteps, &n);
  if (rc < 0) return rc;
  // time_integral.F90:460-465: a replica at its exchange step waits
  if (exchange_step)
    for (int l = 0; l < c->nlane; ++l)
      if (!flg[l] && ls[l].istep + n[l] == exchange_step[l]) flg[l] = 1;
  return rc;
}

extern "C" int tis_get_steps(tis_ctx *c, int64_t *istep) {
  if (!c || !istep) return TIS_E_ARG;
  std::vector<LaneState> ls(c->nlane);
  CK(cudaMemcpyAsync(ls.data(), c->d_lstate.p, ls.size() * sizeof(LaneState), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int l = 0; l < c->nlane; ++l) istep[l] = ls[l].istep;
  return TIS_OK;
}

extern "C" int tis_get_random_number(tis_ctx *c, int64_t istep, int32_t nstep, double *r_boxmuller) {
  if (!c || !r_boxmuller || nstep <= 0 || nstep > 65535) return TIS_E_ARG;
  const size_t n = 3 * (size_t)c->nbead_total * nstep;
  DBuf<double> out;
  CK(out.alloc(n));
  KArgs a = make_args(c, 0, 0, -1);
  ++c->launches;
  CK(noise_launch(c->stream, a, istep, nstep, out.p));
  CK(cudaMemcpyAsync(r_boxmuller, out.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  out.free();
  return TIS_OK;
}

extern "C" int tis_get_rebuild_info(tis_ctx *c, int32_t irep, int64_t *n_rebuild, int64_t *last_step) {
  if (!c || irep < 1 || irep > c->nlane) return TIS_E_ARG;
  LaneState l{};
  CK(cudaMemcpyAsync(&l, c->d_lstate.p + (irep - 1), sizeof(LaneState), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (n_rebuild) *n_rebuild = l.nrebuild;
  if (last_step) *last_step = l.last_rebuild;
  return TIS_OK;
}

// energy_allrep.F90:123-260 + simu_replica_exchange.F90:87-300 +
// time_integral_post.F90:293-349 (labels refresh rlan_const(1) and the
// electrostatic / stack parameters: the kernels read them by label).
namespace {
int exchange_check(tis_ctx *c) {
  if (c->ntop != 1) return fail(c, TIS_E_UNSUPPORTED, "replica exchange needs one topology");
  if (c->nlabel != c->nlane)
    return fail(c, TIS_E_UNSUPPORTED, "a ladder context exchanges through tis_rex_energies and tis_rex_exchange_all");
  return TIS_OK;
}

// The kernels of one exchange, queued without a host wait (u: injected
// uniforms on the host, or NULL for the device's counter-based ones).
int enqueue_exchange(tis_ctx *c, const double *u) {
  const int n = c->nlane;
  // own energies (hbond energies of the last force call reused when valid),
  // then the energies at the partner labels with the partner's beta for the
  // recomputed hbonds (energy_allrep.F90:134,209-216); lanes without a
  // partner are not used
  KArgs a = make_args(c, 0, 0, -1);
  a.reuse_hb = c->hb_energy_valid ? 1 : 0;
  a.elabel = nullptr;
  a.ebeta_lane = nullptr;
  a.out_energy = c->out_energy.p;
  KArgs b = a;
  b.reuse_hb = 0;
  b.elabel = c->elabel.p;
  b.ebeta_lane = c->ebeta.p;
  b.out_energy = c->e_opp.p;
  if (c->par.i_ele != TIS_ELE_EWALD) {
    // the partner labels first, then both passes in one launch (the partner
    // pass recomputes the hbonds in its own scratch)
    ++c->launches;
    CK(rex_launch(c->stream, a, c->rex.p, c->d_rep2lab.p, c->d_lab2rep.p, c->elabel.p, c->ebeta.p));
    b.hb_flag = c->hb_flag2.p; b.hb_ene = c->hb_ene2.p; b.site_exc = c->site_exc2.p;
    b.hb_flag_src = c->hb_flag.p;
    ++c->launches;
    CK(energy_pair_launch(n, c->max_nmp, c->stream, a, b));
  } else {
    ++c->launches;
    CK(energy_kernel_launch(n, c->max_nmp, c->stream, a));
    int rc = ewald_recip(c, a, false);
    if (rc < 0) return rc;
    ++c->launches;
    CK(ewald_energy_launch(c->stream, a));
    ++c->launches;
    CK(rex_launch(c->stream, a, c->rex.p, c->d_rep2lab.p, c->d_lab2rep.p, c->elabel.p, c->ebeta.p));
    ++c->launches;
    CK(energy_kernel_launch(n, c->max_nmp, c->stream, b));
    rc = ewald_recip(c, b, false);
    if (rc < 0) return rc;
    ++c->launches;
    CK(ewald_energy_launch(c->stream, b));
  }
  c->hb_energy_valid = false;
  // the pair alternation does not depend on the decisions, so the host
  // knows this exchange's pair count without reading the device state
  const int npair = (c->idx_pair == 1) ? n / 2 : (n - 1) / 2;
  c->idx_pair = (c->idx_pair == 2) ? 1 : c->idx_pair + 1;
  const double *du = nullptr;
  if (u) {
    if (npair > 0)
      CK(cudaMemcpyAsync(c->rex_u.p, u, (size_t)npair * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    du = c->rex_u.p;
  }
  c->launches += 2;   // the decisions, then the velocity rescale
  CK(rex_exchange_launch(c->stream, a, c->rex.p, c->d_rep2lab.p, c->d_lab2rep.p, c->out_energy.p, c->e_opp.p, du,
                         c->scale.p, c->velo.p));
  return TIS_OK;
}
}  // namespace

extern "C" int tis_replica_exchange(tis_ctx *c, const double *u, int32_t *n_accept) {
  if (!c) return TIS_E_ARG;
  int rc = exchange_check(c);
  if (rc < 0) return rc;
  rc = enqueue_exchange(c, u);
  if (rc < 0) return rc;
  if (n_accept) {   // the only host wait of an exchange
    RexState r;
    CK(cudaMemcpyAsync(&r, c->rex.p, sizeof(RexState), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *n_accept = r.nacc;
  }
  return TIS_OK;
}

// mloop_simulator.F90:123-150, the time-integral loop, for replicas that
// step together: nperiod times [nstep calls of time_integral; with exchange,
// the replica exchange of time_integral_post].  One period's kernels are
// recorded once as a CUDA graph on the context's stream (again when nstep or
// exchange change) and replayed nperiod times; the host waits once, at the
// end, where the replicas' error flags (sticky) are read.  last_ms: the
// device time of the last period's steps (event nodes of the graph).
extern "C" int tis_run(tis_ctx *c, int32_t nperiod, int64_t nstep, int32_t exchange) {
  if (!c || nperiod < 0 || nstep < 1 || nstep > 0x7fffffff) return TIS_E_ARG;
  if (c->bdhi)
    return fail(c, TIS_E_UNSUPPORTED, "tis_run on the Brownian-HI path (its refresh schedule is counted on the host)");
  if (c->noise_nsteps || c->n_unif)
    return fail(c, TIS_E_UNSUPPORTED, "tis_run with injected noise or uniforms (tis_set_noise)");
  exchange = exchange ? 1 : 0;
  if (exchange) {
    const int rc = exchange_check(c);
    if (rc < 0) return rc;
  }
  if (nperiod == 0) return TIS_OK;
  if (!c->g_exec || c->g_nstep != nstep || c->g_exchange != exchange) {
    if (c->g_exec) { cudaGraphExecDestroy(c->g_exec); c->g_exec = nullptr; }
    // recording queues nothing: the host's counters are put back after it
    const long long launches0 = c->launches;
    const int idx_pair0 = c->idx_pair;
    const bool hb_valid0 = c->hb_energy_valid;
    if (!c->g_ev0) { CK(cudaEventCreate(&c->g_ev0)); CK(cudaEventCreate(&c->g_ev1)); }
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    // event nodes around the steps: their last replay times the last period's steps
    cudaError_t er = cudaEventRecordWithFlags(c->g_ev0, c->stream, cudaEventRecordExternal);
    int rc = er == cudaSuccess ? enqueue_steps(c, (int)nstep, nullptr)
                               : fail(c, TIS_E_CUDA, std::string("cudaEventRecordWithFlags: ") + cudaGetErrorString(er));
    if (rc >= 0) {
      er = cudaEventRecordWithFlags(c->g_ev1, c->stream, cudaEventRecordExternal);
      if (er != cudaSuccess) rc = fail(c, TIS_E_CUDA, std::string("cudaEventRecordWithFlags: ") + cudaGetErrorString(er));
    }
    if (rc >= 0 && exchange) {
      c->hb_energy_valid = true;   // the steps' last force call left the hbond energies
      rc = enqueue_exchange(c, nullptr);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->g_launches = c->launches - launches0;
    c->launches = launches0;
    c->idx_pair = idx_pair0;
    c->hb_energy_valid = hb_valid0;
    if (rc < 0 || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return rc < 0 ? rc : fail(c, TIS_E_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
    }
    const cudaError_t ei = cudaGraphInstantiate(&c->g_exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
      c->g_exec = nullptr;
      return fail(c, TIS_E_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ei));
    }
    c->g_nstep = nstep;
    c->g_exchange = exchange;
  }
  for (int p = 0; p < nperiod; ++p) CK(cudaGraphLaunch(c->g_exec, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c->g_ev0, c->g_ev1));
  c->last_ms = ms;
  c->launches += (long long)nperiod * c->g_launches;
  c->hb_energy_valid = !exchange;
  if (exchange)
    for (int p = 0; p < nperiod; ++p) c->idx_pair = (c->idx_pair == 2) ? 1 : c->idx_pair + 1;
  return check_lanes(c);
}

extern "C" int tis_get_labels(tis_ctx *c, int32_t *rep2lab) {
  if (!c || !rep2lab) return TIS_E_ARG;
  std::vector<LaneState> ls(c->nlane);
  CK(cudaMemcpyAsync(ls.data(), c->d_lstate.p, ls.size() * sizeof(LaneState), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < c->nlane; ++k) rep2lab[k] = ls[k].label + 1;
  return TIS_OK;
}

// ------------------------------------------------ ladder split over ranks
// simu_replica_exchange.F90:121-267 for one exchange of a whole ladder on
// the host, after every rank's replica_energy has been gathered
// (time_integral_post.F90:279): the pairs of this exchange's odd/even
// alternation in label order, the k-th taking uniform u[k]; an accepted
// pair swaps the labels of its two replicas and rescales their velocities.
extern "C" int tis_rex_decide(int32_t nrep_all, const double *tempk_all, int32_t idx_pair,
                              const double *replica_energy, const double *u, int32_t *rep2lab, double *vscale,
                              int32_t *n_accept) {
  if (nrep_all <= 0 || !tempk_all || !replica_energy || !u || !rep2lab || (idx_pair != 1 && idx_pair != 2))
    return TIS_E_ARG;
  const int n = nrep_all;
  std::vector<int> lab2rep(n, -1);
  for (int r = 0; r < n; ++r) {
    const int l = rep2lab[r];
    if (l < 1 || l > n || lab2rep[l - 1] >= 0) return TIS_E_ARG;
    lab2rep[l - 1] = r;
  }
  if (vscale) for (int r = 0; r < n; ++r) vscale[r] = 0.0;
  int k = 0, nacc = 0;
  for (int li = 1; li <= n; ++li) {
    const int lj = rex_pair(li, n, idx_pair);
    if (lj < li) continue;
    const int ri = lab2rep[li - 1], rj = lab2rep[lj - 1];
    const double tm = tempk_all[li - 1], tn = tempk_all[lj - 1];
    const double pim = replica_energy[2 * ri], pin = replica_energy[2 * ri + 1];
    const double pjn = replica_energy[2 * rj], pjm = replica_energy[2 * rj + 1];
    const double delta = ((pjm - pim) / tm - (pjn - pin) / tn) / BOLTZ_KCAL_MOL;
    const double uu = u[k++];
    if (delta < 0.0e0 || uu <= std::exp(-delta)) {
      rep2lab[ri] = lj; rep2lab[rj] = li;
      lab2rep[li - 1] = rj; lab2rep[lj - 1] = ri;
      const double sf = std::sqrt(tn / tm);
      if (vscale) { vscale[ri] = sf; vscale[rj] = -sf; }
      ++nacc;
    }
  }
  if (n_accept) *n_accept = nacc;
  return TIS_OK;
}

extern "C" int tis_rex_energies(tis_ctx *c, double *replica_energy) {
  if (!c || !replica_energy) return TIS_E_ARG;
  if (c->g_rep2lab.empty()) return fail(c, TIS_E_UNSUPPORTED, "tis_rex_energies: not a ladder context");
  // energy_allrep.F90:123-217: the own label's energy (hbond energies of the
  // last force call reused), then the partner label's with its beta
  std::vector<double> E, E2;
  int rc = run_energy(c, -1, nullptr, c->hb_energy_valid, c->beta_global, E);
  if (rc < 0) return rc;
  std::vector<int> elab(c->nlane);
  std::vector<double> beta(c->nlane);
  for (int l = 0; l < c->nlane; ++l) {
    const int lo = rex_pair(c->g_rep2lab[c->rep_first + l] + 1, c->nlabel, c->idx_pair);
    elab[l] = lo ? lo - 1 : -1;
    beta[l] = lo ? 1.0e0 / (c->lab_T[lo - 1] * BOLTZ_KCAL_MOL) : c->beta_global;
  }
  rc = run_energy(c, -1, elab.data(), false, c->beta_global, E2, beta.data());
  if (rc < 0) return rc;
  c->hb_energy_valid = false;
  for (int l = 0; l < c->nlane; ++l) {
    replica_energy[2 * l] = E[(size_t)l * N_ETYPE + TIS_E_TOTAL - 1];
    replica_energy[2 * l + 1] = elab[l] >= 0 ? E2[(size_t)l * N_ETYPE + TIS_E_TOTAL - 1] : 0.0;
  }
  return check_lanes(c);
}

extern "C" int tis_rex_exchange_all(tis_ctx *c, const double *replica_energy_all, const double *u,
                                    int32_t *n_accept) {
  if (!c || !replica_energy_all) return TIS_E_ARG;
  if (c->g_rep2lab.empty()) return fail(c, TIS_E_UNSUPPORTED, "tis_rex_exchange_all: not a ladder context");
  const int n = c->nlabel;
  int npair = 0;
  for (int li = 1; li <= n; ++li) npair += rex_pair(li, n, c->idx_pair) > li;
  std::vector<double> uu(std::max(npair, 1));
  if (u) {
    for (int k = 0; k < npair; ++k) uu[k] = u[k];
  } else {   // the device exchange's counter-based uniforms (same seed on every rank)
    for (int k = 0; k < npair; ++k) {
      const unsigned long long ctr = c->g_counter + (unsigned long long)k;
      const U4 o = philox4x32(U4{(uint32_t)ctr, (uint32_t)(ctr >> 32), 0x52454D44u, 0u}, (uint32_t)c->par.seed,
                              (uint32_t)(c->par.seed >> 32));
      uu[k] = u01_open0(o.x) - 2.3283064365386963e-10;
    }
    c->g_counter += (unsigned long long)npair;
  }
  std::vector<int> r2l(n);
  for (int g = 0; g < n; ++g) r2l[g] = c->g_rep2lab[g] + 1;
  std::vector<double> vs(n);
  int nacc = 0;
  int rc = tis_rex_decide(n, c->lab_T.data(), c->idx_pair, replica_energy_all, uu.data(), r2l.data(), vs.data(),
                          &nacc);
  if (rc < 0) return fail(c, rc, "tis_rex_exchange_all: inconsistent label maps");
  for (int g = 0; g < n; ++g) { c->g_rep2lab[g] = r2l[g] - 1; c->g_lab2rep[r2l[g] - 1] = g; }
  c->idx_pair = (c->idx_pair == 2) ? 1 : c->idx_pair + 1;
  // beta_hbond15 of the last replica's label (simu_set_dtrna.F90:58)
  c->beta_global = 1.0e0 / (c->lab_T[c->g_rep2lab[n - 1]] * BOLTZ_KCAL_MOL);
  // the local replicas' labels and velocities
  std::vector<LaneState> ls(c->nlane);
  CK(cudaMemcpyAsync(ls.data(), c->d_lstate.p, ls.size() * sizeof(LaneState), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::vector<double> sc(c->nlane);
  for (int l = 0; l < c->nlane; ++l) {
    ls[l].label = c->g_rep2lab[c->rep_first + l];
    c->rep2lab[l] = ls[l].label;
    sc[l] = vs[c->rep_first + l];
  }
  CK(cudaMemcpyAsync(c->d_lstate.p, ls.data(), ls.size() * sizeof(LaneState), cudaMemcpyHostToDevice, c->stream));
  RexState r{};
  r.beta_global = c->beta_global;
  r.counter = c->g_counter;
  r.idx_pair = c->idx_pair;
  r.nacc = nacc;
  CK(cudaMemcpyAsync(c->rex.p, &r, sizeof(RexState), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->scale.p, sc.data(), sc.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  KArgs a = make_args(c, 0, 0, -1);
  ++c->launches;
  CK(vscale_launch(c->stream, a, c->scale.p, c->velo.p));
  CK(cudaStreamSynchronize(c->stream));
  if (n_accept) *n_accept = nacc;
  return TIS_OK;
}

extern "C" int tis_status(tis_ctx *c, tis_status_t *st) {
  if (!c || !st) return TIS_E_ARG;
  std::vector<LaneState> ls(c->nlane);
  CK(cudaMemcpy(ls.data(), c->d_lstate.p, ls.size() * sizeof(LaneState), cudaMemcpyDeviceToHost));
  std::memset(st, 0, sizeof(*st));
  st->step = ls[0].istep;
  for (int i = 0; i < c->nlane; ++i) {
    st->n_rebuild += ls[i].nrebuild;
    st->n_clamp += ls[i].nclamp;
    st->list_overflow |= (ls[i].flags & LF_OVERFLOW) ? 1 : 0;
    st->nan_seen |= (ls[i].flags & LF_NAN) ? 1 : 0;
    st->exv_pairs_max = std::max(st->exv_pairs_max, ls[i].nexv);
    st->ele_pairs_max = std::max(st->ele_pairs_max, ls[i].nele);
  }
  st->ctas_per_lane = c->pair ? 2 : 1;
  st->threads_per_cta = c->pair ? 512 : c->threads;
  st->group = c->group;
  st->noise_sweep = c->noise_sweep;
  st->lane_order = c->order;
  st->sweep = c->sweep;
  st->launch_source = c->launch_source;
  st->wait_timeout = c->wait_timeout;
  st->not_spd = c->not_spd;
  st->last_error = c->last_error;
  return TIS_OK;
}

extern "C" double tis_last_step_ms(tis_ctx *c) { return c ? c->last_ms : -1.0; }

extern "C" int tis_timer(tis_ctx *c, int32_t op, double *ms) {
  if (!c) return TIS_E_ARG;
  if (!c->tev0) { CK(cudaEventCreate(&c->tev0)); CK(cudaEventCreate(&c->tev1)); }
  if (op == 0) { CK(cudaEventRecord(c->tev0, c->stream)); return TIS_OK; }
  if (op != 1 || !ms) return TIS_E_ARG;
  CK(cudaEventRecord(c->tev1, c->stream));
  CK(cudaEventSynchronize(c->tev1));
  float f = 0.f;
  CK(cudaEventElapsedTime(&f, c->tev0, c->tev1));
  *ms = f;
  return TIS_OK;
}

extern "C" const char *tis_last_error(const tis_ctx *c) { return c ? c->err.c_str() : "null context"; }

extern "C" int64_t tis_launch_count(const tis_ctx *c) { return c ? (int64_t)c->launches : -1; }

extern "C" int tis_get_hydro_tensors(tis_ctx *c, int32_t irep, double *diffuse, double *random) {
  if (!c || irep < 1 || irep > c->nlane) return TIS_E_ARG;
  if (!c->bdhi) return fail(c, TIS_E_UNSUPPORTED, "no hydrodynamic tensors: not a Brownian-HI context");
  const LaneDesc &L = c->lanes[irep - 1];
  const size_t n = 3 * (size_t)c->lane_nmp[irep - 1];
  std::vector<double> buf(n * n);
  std::vector<float> fbuf;
  // device storage is row-major; the reference arrays are column-major.
  // Mixed precision keeps D in FP32 only (rows padded to a multiple of 4);
  // the factor's upper part is never stored on the device (the reference's
  // random_tensor holds zeros there).
  for (int which = 0; which < 2; ++which) {
    double *out = which == 0 ? diffuse : random;
    if (!out) continue;
    if (which == 0 && c->bd_D32.p) {
      const size_t ld = (n + 3) / 4 * 4;
      fbuf.resize(n * ld);
      CK(cudaMemcpy(fbuf.data(), c->bd_D32.p + L.bd32, n * ld * sizeof(float), cudaMemcpyDeviceToHost));
      for (size_t r = 0; r < n; ++r)
        for (size_t col = 0; col < n; ++col) buf[r * n + col] = fbuf[r * ld + col];
    } else {
      CK(cudaMemcpy(buf.data(), (which == 0 ? c->bd_D.p : c->bd_L.p) + L.bd0, n * n * sizeof(double),
                    cudaMemcpyDeviceToHost));
    }
    for (size_t r = 0; r < n; ++r)
      for (size_t col = 0; col < n; ++col) out[col * n + r] = (which == 1 && col > r) ? 0.0 : buf[r * n + col];
  }
  return TIS_OK;
}

// ------------------------------------------------ force without allocation
// tis_force_sumup_static: neighbour lists + forces of one replica for
// caller-owned device coordinates, with every per-call buffer (lane
// descriptor and scalar state, coordinates, list bit matrices, mirror
// indices, interaction slots, hbond flags/energies, site counters) carved
// out of one file-scope device array instead of the context's buffers.
// The array is STATIC_SCRATCH_BYTES long, lives on every GPU that loads the
// library until process exit, and is shared by all calls on that GPU.
namespace {

constexpr size_t STATIC_SCRATCH_BYTES = (size_t)1 << 20;   // 1 MiB per GPU
constexpr int STATIC_MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_static_scratch[STATIC_SCRATCH_BYTES];

std::mutex g_static_mu;
unsigned char *g_static_ptr[STATIC_MAX_DEVICES] = {};

// Set-up, once per device with that device current: the address of the
// array on the current device.  Runs inside the first call on each device.
// The cached address belongs to the device's primary context, which the
// CUDA runtime keeps for the whole process; a process that resets a device
// (cudaDeviceReset) must not call tis_force_sumup_static on it afterwards.
int static_scratch_ptr(tis_ctx *c, unsigned char **out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= STATIC_MAX_DEVICES) return fail(c, TIS_E_UNSUPPORTED, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p)
      return fail(c, TIS_E_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
    g_static_ptr[dev] = (unsigned char *)p;
  }
  *out = g_static_ptr[dev];
  return TIS_OK;
}

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

// Byte offsets of the per-call buffers inside the static array.
struct StaticLayout {
  size_t lanes, lstate, xyz, pxyz, velo, accel, dxyz, p0xyz, mask, mirror, slots, hb_flag, hb_ene, site_exc, total;
};

StaticLayout static_layout(const tis_ctx *c, int lane) {
  const TopDesc &T = c->tops[c->lanes[lane].top];
  const size_t N = (size_t)T.nmp, W = (N + 31) / 32;
  const size_t real_size = c->par.precision == TIS_PREC_MIXED ? sizeof(float) : sizeof(double);
  StaticLayout s{};
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o += align256(std::max<size_t>(bytes, 1)); return at; };
  s.lanes = take((size_t)c->nlane * sizeof(LaneDesc));
  s.lstate = take((size_t)c->nlane * sizeof(LaneState));
  s.xyz = take(3 * N * sizeof(double));
  s.pxyz = take(3 * N * sizeof(double));
  s.velo = take(3 * N * sizeof(double));
  s.accel = take(3 * N * sizeof(double));
  s.dxyz = take(3 * N * sizeof(double));
  s.p0xyz = take(c->par.i_periodic == 1 ? 3 * N * sizeof(double) : 1);
  s.mask = take(2 * N * W * sizeof(uint32_t));
  s.mirror = take(c->par.i_periodic == 1 ? N * N : 1);
  s.slots = take((size_t)T.nslot * 3 * real_size);
  s.hb_flag = take((size_t)T.nhb);
  s.hb_ene = take((size_t)T.nhb * sizeof(double));
  s.site_exc = take((size_t)T.nsite * sizeof(int));
  s.total = o;
  return s;
}

}  // namespace

extern "C" int tis_force_sumup_static(tis_ctx *c, int32_t irep, const double *xyz_dev, double *force_dev) {
  if (!c || irep < 1 || irep > c->nlane || !xyz_dev || !force_dev) return TIS_E_ARG;
  // Brownian-HI contexts never size the lane kernel's shared memory and
  // evaluate FENE / WCA records, not the DT15 terms this call computes
  if (c->bdhi)
    return fail(c, TIS_E_UNSUPPORTED, "tis_force_sumup_static: not available on a Brownian-HI context");
  if (c->par.i_ele == TIS_ELE_EWALD)
    return fail(c, TIS_E_UNSUPPORTED, "tis_force_sumup_static: Ewald needs the context's reciprocal-space buffers");
  const int lane = irep - 1;
  const StaticLayout lay = static_layout(c, lane);
  if (lay.total > STATIC_SCRATCH_BYTES)
    return fail(c, TIS_E_UNSUPPORTED,
                "tis_force_sumup_static: replica " + std::to_string(irep) + " needs " + std::to_string(lay.total) +
                    " bytes of scratch, more than the " + std::to_string(STATIC_SCRATCH_BYTES) +
                    "-byte static area");
  unsigned char *base = nullptr;
  int rc = static_scratch_ptr(c, &base);
  if (rc < 0) return rc;
  const size_t N = (size_t)c->lane_nmp[lane];
  // The array keeps the previous call's contents: start from zeros.
  CK(cudaMemsetAsync(base, 0, lay.total, c->stream));
  // this replica's descriptor with every offset rebased onto the static array
  LaneDesc L = c->lanes[lane];
  L.state0 = 0; L.mask0 = 0; L.mirror0 = 0; L.slot0 = 0; L.hb0 = 0; L.site0 = 0;
  CK(cudaMemcpyAsync(base + lay.lanes + lane * sizeof(LaneDesc), &L, sizeof(LaneDesc), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaMemcpyAsync(base + lay.lstate + lane * sizeof(LaneState), c->d_lstate.p + lane, sizeof(LaneState),
                     cudaMemcpyDeviceToDevice, c->stream));
  // the context's sticky flags (an earlier NAN, overflow or exhausted noise)
  // do not belong to this call
  CK(cudaMemsetAsync(base + lay.lstate + lane * sizeof(LaneState) + offsetof(LaneState, flags), 0, sizeof(int),
                     c->stream));
  CK(cudaMemcpyAsync(base + lay.xyz, xyz_dev, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(base + lay.pxyz, xyz_dev, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  LaneState before{};
  CK(cudaMemcpyAsync(&before, c->d_lstate.p + lane, sizeof(LaneState), cudaMemcpyDeviceToHost, c->stream));

  KArgs a = make_args(c, KM_NEIGHBOR, 0, lane);
  a.lanes = (const LaneDesc *)(base + lay.lanes);
  a.lstate = (LaneState *)(base + lay.lstate);
  a.xyz = (double *)(base + lay.xyz); a.pxyz = (double *)(base + lay.pxyz);
  a.velo = (double *)(base + lay.velo); a.accel = (double *)(base + lay.accel); a.dxyz = (double *)(base + lay.dxyz);
  a.p0xyz = (double *)(base + lay.p0xyz);
  a.mask = (uint32_t *)(base + lay.mask);
  a.mirror = (uint8_t *)(base + lay.mirror);
  a.slots = (decltype(a.slots))(base + lay.slots);
  a.hb_flag = (uint8_t *)(base + lay.hb_flag);
  a.hb_ene = (double *)(base + lay.hb_ene);
  a.site_exc = (int *)(base + lay.site_exc);
  a.out_force = force_dev;
  rc = launch_lane(c, a);
  if (rc < 0) return rc;
  a.mode = KM_FORCE;
  rc = launch_lane(c, a);
  if (rc < 0) return rc;
  LaneState after{};
  CK(cudaMemcpyAsync(&after, base + lay.lstate + lane * sizeof(LaneState), sizeof(LaneState), cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (after.flags & LF_NAN) return fail(c, TIS_E_NAN, "non-finite force in lane " + std::to_string(irep));
  if (after.flags & LF_PMF) return fail(c, TIS_E_PMF_RANGE, "Mg-P pair below the PMF table in lane " + std::to_string(irep));
  if (after.flags & LF_OVERFLOW) return fail(c, TIS_E_LIST_OVERFLOW, "hbond site list overflow");
  if (after.flags & (LF_UNIF_EXHAUSTED | LF_NOISE_EXHAUSTED))
    return fail(c, TIS_E_NOISE_EXHAUSTED, "injected noise or uniforms exhausted");
  return (int)std::min<long long>(std::max<long long>(after.nclamp - before.nclamp, 0), 0x7fffffff);
}
