// tis_oracle.cpp -- CPU FP64 restatement of the TIS (Hori-Lab/TIS, Fortran)
// force-and-integrate path.  TEST INFRASTRUCTURE ONLY: this file is the
// checker that the CUDA path is compared against.  Nothing in the product
// library links, loads or calls it.
//
// Parity status: UNPINNED against reference outputs.  The reference is
// Fortran, this image has no Fortran compiler, and the reference ships no
// golden vectors for this path.  The restatement is pinned instead by the
// identities the reference itself uses as checks: F = -grad E by central
// differences (src/simu_checkforce.F90:79-140), Ewald against a direct
// lattice sum (utility/coulomb_energy_exact.F90), and analytic single
// interaction cases.
//
// Every routine cites the reference lines it follows.  Loop order, the
// order of floating-point operations and the order of accumulation into
// force_mp follow the Fortran (compiled here with -ffp-contract=off).
// Transcendentals come from glibc libm (the reference uses the Fortran
// compiler's intrinsics; that boundary is unpinned).

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>

#include "../include/tis_b200.h"

namespace {

// ---- const_physical.F90:9-38 ------------------------------------------
const double F_PI = 3.14159265358979323846264338e0;
const double F_2PI = 2.0 * F_PI;
const double EPSI_0 = 8.854187817e-12;
const double ELE = 1.6021766208e-19;
const double BOLTZ_J = 1.38064852e-23;
const double N_AVO = 6.022140857e23;
const double KCAL2JOUL = 4184.0;
const double JOUL2KCAL = 1.0 / KCAL2JOUL;
const double JOUL2KCAL_MOL = JOUL2KCAL * N_AVO;
const double BOLTZ_KCAL_MOL = BOLTZ_J * JOUL2KCAL_MOL;
const double DE_MAX = 50.0;
const double ZERO_JUDGE = 1.0e-6;
const double HIGH_ENERGY = 1.0e10;
// cos(0.57/180.0 * F_PI): 0.57/180.0 is a default-real (single) quotient.
const double MAX_ANG_ABSCOS_HBOND15 = std::cos((double)(0.57f / 180.0f) * F_PI);
const double MAX_DIH_ABSCOS_HBOND15 = MAX_ANG_ABSCOS_HBOND15;

inline double sq(double x) { return x * x; }
// dot_product of 3-vectors as gfortran evaluates it: ((a1b1 + a2b2) + a3b3)
inline double dot3(const double *a, const double *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
inline double norm2_3(const double *a) { return std::sqrt(dot3(a, a)); }

struct Label {           // per temperature label: simu_ele_set / simu_set_dtrna
  double tempk;
  double ek, coef, cdist;
  double zp = 0.0;             // i_charge = 1: phosphate charge -zp (simu_ele_set.F90:107-166)
  std::vector<double> pmf_e, pmf_f;   // pmfdh_energy / pmfdh_force (simu_ele_set.F90:231-253)
  std::vector<double> st_u0;   // coef_dtrna_st(0, ist, grep)
};

struct Rep {
  std::vector<double> xyz, pxyz, velo, accel, force, dxyz;
  std::vector<int> iexv2mp;       // (3, nexv) 1-based, col 3 = imirror
  std::vector<int> iele2mp;       // (4, nele)
  std::vector<double> coef_ele;
  std::vector<int> ineigh2hb;     // 1-based hb indices
  std::vector<char> hb_status;
  std::vector<double> ene_hb;
  std::vector<char> st_status;
  std::vector<double> for_hb;     // (3, 6, nhb)
  std::vector<int> hbsite_excess;
  int label = 1;                  // rep2lab
  long istep = 0;                 // time_integral calls so far
  std::vector<double> unif;       // injected uniforms for valence pruning
  size_t upos = 0;
  bool unif_exhausted = false;
  long nclamp = 0;
  long nrebuild = 0;
  long last_rebuild = -1;          // istep of the last neighbour rebuild
  int pmf_range = 0;              // a Mg-P pair below the PMF table's first point
  std::vector<double> hD, hL;     // Brownian-HI: diffuse_tensor, random_tensor (3N x 3N, column-major)
  int not_spd = 0;
};

} // namespace

struct orc_ctx {
  // topology (0-based copies)
  int nmp = 0, nunit = 0;
  std::vector<int> lunit2mp, iclass_unit, imp2type, imp2unit, iclass_mp;
  std::vector<double> cmass, fric, exv_radius, exv_epsilon, rcmass;
  int ncharge = 0;
  std::vector<int> icharge2mp;
  std::vector<int> lmp2charge;
  std::vector<double> coef_charge;
  std::vector<char> q_kind;        // 1: phosphate whose charge is -Zp of the label (i_charge = 1)
  int n_mg = 0;                    // num_ion(IONTYPE%MG)
  bool dt19 = false;               // i_dtrna_model = 2019
  std::vector<double> pmf;         // inpmf%pmf(:, MG_P)
  int nbd = 0; std::vector<int> ibd2mp; std::vector<double> bd_nat, coef_bd;
  int nba = 0; std::vector<int> iba2mp; std::vector<double> ba_nat, coef_ba;
  int nst = 0; std::vector<int> st2mp; std::vector<double> st_nat, st_coef, st_hsTm;
  int nhb = 0; std::vector<int> hb2mp; std::vector<double> hb_nat, hb_coef; std::vector<int> hb2site;
  std::vector<char> hb_tert;        // flg_hb_tertiary (read_nativeinfo.F90:606-613)
  int nhbsite = 0; std::vector<int> nvalence;
  std::vector<std::vector<int>> hb_at_site;   // static per-site hb lists (ascending ihb)
  int nfene = 0; std::vector<int> fene2mp; std::vector<double> fene_nat, coef_fene, dist2_fene;
  int nwca = 0; std::vector<int> wca2mp; std::vector<double> wca_nat, coef_wca;
  std::vector<double> radius;      // var_struct radius: hydrodynamic radius per bead (Brownian-HI)
  int ntst = 0; std::vector<int> tst2mp; std::vector<double> tst_nat, tst_coef;
  std::vector<int> tst2st;         // (2, ntst) 0-based secondary stack of each side, -1: none
  std::vector<char> tst_excl;      // (2, ntst) after mloop_dtrna.F90:74-140
  tis_params par;
  // derived
  std::vector<double> rneighbordist2_unit;   // (nunit, nunit)
  double psizeh[3];
  double d_mirror[27][3];
  std::vector<double> hb_neigh_dist2;
  double tstep2 = 0, tsteph = 0;
  double beta_hbond15 = 0;
  // Ewald
  int ewld_f_n = 0;
  std::vector<double> ewld_f_rlv, ewld_f_coef;
  double ewld_s_coef = 0;
  // replicas and labels
  int nrep = 0;
  std::vector<Rep> rep;
  std::vector<Label> lab;          // lab2val(l, TEMP) for l = 1..nrep
  std::vector<int> lab2rep;
  int idx_pair = 1;                // var_replica.F90 set_forward alternation
  // noise injection
  std::vector<double> noise;       // (3, nmp, nrep, nsteps)
  int noise_nsteps = 0;
  int noise_pos = 0;
  bool noise_exhausted = false;
};

namespace {

// simu_ele_set.F90:46-226 (i_temp_independent = 0, i_charge = 0 path).
void ele_set(const orc_ctx &c, Label &L) {
  const double MM_A = 87.740e0, MM_B = -0.4008e0, MM_C = 9.398e-4, MM_D = -1.410e-6;
  double ek = 0.0;
  if (c.par.i_diele == 0) {
    ek = c.par.diele_water;
  } else {
    double Tc = L.tempk - 273.15e0;
    ek = MM_A + MM_B * Tc + MM_C * Tc * Tc + MM_D * Tc * Tc * Tc;
  }
  L.ek = ek;
  // simu_ele_set.F90:107-166: Manning condensation; with Mg in the DT19
  // model the condensed fraction theta solves the two-ion balance
  if (c.par.i_charge == 1) {
    const double lb = ELE * ELE / (4.0e0 * F_PI * EPSI_0 * ek * BOLTZ_J * L.tempk) * 1.0e10;
    const double b = c.par.length_per_unit_P;
    if (c.dt19 && c.n_mg > 0) {
      const double xi = lb / b, b3 = b * b * b;
      const double conc_Mg = c.n_mg / (N_AVO * 1.0e-27 * c.par.psize[0] * c.par.psize[1] * c.par.psize[2]);
      const double v1 = 4 * F_PI * b3 * (xi - 1.0e0) * 2;
      const double v2 = 4 * F_PI * b3 * (xi - 0.5e0) * (2 + 1);
      const double c1v1 = (N_AVO * 1.0e-27) * c.par.ionic_strength * v1;
      const double c2v2 = (N_AVO * 1.0e-27) * conc_Mg * v2;
      const double c1v1_2 = c1v1 * c1v1;
      const double theta = (-c1v1_2 + std::sqrt(c1v1_2 * c1v1_2 + 8.0e0 * c1v1_2 * c2v2 * (1.0e0 - 1.0e0 / xi))) /
                           (4.0e0 * c2v2);
      L.zp = 1.0 - theta;
    } else {
      L.zp = b / lb;
    }
  }
  L.coef = JOUL2KCAL_MOL * 1.0e10 * (ELE * ELE) / (4.0e0 * F_PI * EPSI_0 * ek);
  L.cdist = 1.0e10 * std::sqrt((1.0e-3 * EPSI_0 * ek * BOLTZ_J) / (2.0 * N_AVO * (ELE * ELE))) *
            std::sqrt(L.tempk / c.par.ionic_strength);
  // simu_ele_set.F90:231-253: the Mg-P table, PMF switched to DH beyond
  // pmf_merge; the force of the last point is 0 (the reference never sets it)
  L.pmf_e.clear(); L.pmf_f.clear();
  if (c.dt19 && c.n_mg > 0 && !c.pmf.empty()) {
    const int nb = c.par.pmf_nbin;
    L.pmf_e.assign(nb, 0.0); L.pmf_f.assign(nb, 0.0);
    for (int ib = 0; ib < nb; ++ib) {
      const double r = c.par.pmf_rmin + c.par.pmf_rbin * (double)ib;
      const double DH = JOUL2KCAL_MOL * 1.0e10 * (ELE * ELE) / (4.0e0 * F_PI * EPSI_0 * ek) * 2.0 * (-L.zp) *
                        std::exp(-r / L.cdist) / r;
      const double e_add = (DH - c.pmf[ib]) * std::exp(-(c.par.pmf_rmerge * c.par.pmf_rmerge) / (r * r));
      L.pmf_e[ib] = c.pmf[ib] + e_add;
    }
    const double rbininv = 1.0 / c.par.pmf_rbin;
    for (int ib = 0; ib + 1 < nb; ++ib) L.pmf_f[ib] = -rbininv * (L.pmf_e[ib + 1] - L.pmf_e[ib]);
  }
}

// charge of charge entry ic for label L (coef_charge(ic, grep))
inline double qch(const orc_ctx &c, const Label &L, int ic) {
  return c.q_kind[ic] ? -L.zp : c.coef_charge[ic];
}

bool is_mg_p(const orc_ctx &c, int i1, int i2) {
  const int t1 = c.imp2type[i1], t2 = c.imp2type[i2];
  return (t1 == TIS_MP_RNA_PHOS && t2 == TIS_MP_ION_MG) || (t1 == TIS_MP_ION_MG && t2 == TIS_MP_RNA_PHOS);
}

// force_ele_DH.F90:87-100 / energy_ele_DH.F90:77-95: 0-based bin of a Mg-P
// distance; below the first point the reference stops, here the pair takes
// bin 0 and the replica records it
int pmf_bin(const orc_ctx &c, Rep &r, double dist1) {
  if (!(dist1 >= c.par.pmf_rmin)) { r.pmf_range = 1; return 0; }
  int ib = (int)std::floor((dist1 - c.par.pmf_rmin) * (1.0 / c.par.pmf_rbin));
  return std::min(ib, c.par.pmf_nbin - 1);
}

// simu_set_dtrna.F90:43-58 (i_temp_independent = 0)
void set_dtrna(orc_ctx &c, Label &L) {
  L.st_u0.assign(c.nst, 0.0);
  for (int ist = 0; ist < c.nst; ++ist) {
    double h = c.st_hsTm[3 * ist + 0], s = c.st_hsTm[3 * ist + 1], Tm = c.st_hsTm[3 * ist + 2];
    L.st_u0[ist] = -h + BOLTZ_KCAL_MOL * (L.tempk - Tm) * s;
  }
}

// simu_para2.F90: every replica in order; the scalar beta_hbond15 keeps the
// value set for the last replica (simu_set_dtrna.F90:58).
void para2(orc_ctx &c) {
  if (c.nrep > 0) {
    const Label &L = c.lab[c.rep[c.nrep - 1].label - 1];
    c.beta_hbond15 = 1.0e0 / (L.tempk * BOLTZ_KCAL_MOL);
  }
}

// util_pbneighbor.F90:4-39
inline void pbneighbor(const orc_ctx &c, double *v, int *imirror) {
  int imi[3];
  for (int ix = 0; ix < 3; ++ix) {
    if (v[ix] > c.psizeh[ix]) { v[ix] = v[ix] - c.par.psize[ix]; imi[ix] = 0; }
    else if (v[ix] < -c.psizeh[ix]) { v[ix] = v[ix] + c.par.psize[ix]; imi[ix] = 1; }
    else imi[ix] = 2;
  }
  if (imirror) *imirror = 9 * imi[0] + 3 * imi[1] + imi[2] + 1;
}

// util_periodic.F90:4-39
void util_periodic(orc_ctx &c, Rep &r) {
  double pwide[3], pmax[3], pmin[3];
  for (int i = 0; i < 3; ++i) {
    pwide[i] = c.par.psize[i]; pmax[i] = 0.5 * pwide[i]; pmin[i] = -0.5 * pwide[i];
  }
  for (int imp = 0; imp < c.nmp; ++imp)
    for (int ix = 0; ix < 3; ++ix) {
      double tx = r.pxyz[3 * imp + ix];
      if (tx > pmax[ix]) tx = tx - pwide[ix] * (double)((long)((tx - pmax[ix]) / pwide[ix]) + 1);
      else if (tx < pmin[ix]) tx = tx + pwide[ix] * (double)((long)((pmin[ix] - tx) / pwide[ix]) + 1);
      r.pxyz[3 * imp + ix] = tx;
    }
}

int nsep_of(const orc_ctx &c, int imp) {
  switch (c.imp2type[imp]) {
    case TIS_MP_RNA_PHOS: return c.par.n_sep_nlocal_P;
    case TIS_MP_RNA_SUGAR: return c.par.n_sep_nlocal_S;
    case TIS_MP_RNA_BASE: return c.par.n_sep_nlocal_B;
    default: return -1;
  }
}

// neighbor_list.F90:49-90 + neighbor_assign.F90:481-559 + neighbor_sort
// (single list type EXV_DT15, so the type sort keeps generation order) +
// neighbor_assign.F90:742-770 (mirror index).  neighbor_pre marks every
// unit pair that contains an ion or that is intra-unit as neighbouring; for
// distinct RNA units it compares centre distances (neighbor_pre.F90:225-252).
void neighbor_exv(orc_ctx &c, Rep &r) {
  const bool peri = c.par.i_periodic == 1;
  const double *X = peri ? r.pxyz.data() : r.xyz.data();
  // neighbor_pre.F90:174-252
  std::vector<double> cm(3 * c.nunit, 0.0), maxdist(c.nunit, 0.0);
  for (int u = 0; u < c.nunit; ++u) {
    if (c.iclass_unit[u] == TIS_CLASS_ION) continue;
    int is = c.lunit2mp[2 * u] - 1, ie = c.lunit2mp[2 * u + 1] - 1;
    double sx = 0, sy = 0, sz = 0;
    for (int imp = is; imp <= ie; ++imp) {
      sx += r.xyz[3 * imp]; sy += r.xyz[3 * imp + 1]; sz += r.xyz[3 * imp + 2];
    }
    double n = (double)(ie - is + 1);
    cm[3 * u] = sx / n; cm[3 * u + 1] = sy / n; cm[3 * u + 2] = sz / n;
    double md = 0.0;
    for (int imp = is; imp <= ie; ++imp) {
      double d2 = sq(r.xyz[3 * imp] - cm[3 * u]) + sq(r.xyz[3 * imp + 1] - cm[3 * u + 1]) +
                  sq(r.xyz[3 * imp + 2] - cm[3 * u + 2]);
      if (d2 > md) md = d2;
    }
    maxdist[u] = std::sqrt(md);
  }
  if (peri) {
    for (int u = 0; u < c.nunit; ++u) {
      if (c.iclass_unit[u] == TIS_CLASS_ION) continue;
      for (int ix = 0; ix < 3; ++ix) {
        double pw = c.par.psize[ix], pmx = 0.5 * pw, pmn = -0.5 * pw;
        double tx = cm[3 * u + ix];
        if (tx > pmx) tx = tx - pw * (double)((long)((tx - pmx) / pw) + 1);
        else if (tx < pmn) tx = tx + pw * (double)((long)((pmn - tx) / pw) + 1);
        cm[3 * u + ix] = tx;
      }
    }
  }
  std::vector<int> neigh_unit(c.nunit * c.nunit, 0);
  for (int u = 0; u < c.nunit; ++u)
    for (int v = u; v < c.nunit; ++v) {
      int val = 0;
      if (c.iclass_unit[u] == TIS_CLASS_ION || c.iclass_unit[v] == TIS_CLASS_ION) val = 1;
      else if (u == v) val = 1;
      else {
        double v21[3] = {cm[3 * v] - cm[3 * u], cm[3 * v + 1] - cm[3 * u + 1], cm[3 * v + 2] - cm[3 * u + 2]};
        if (peri) pbneighbor(c, v21, nullptr);
        if (norm2_3(v21) < maxdist[u] + maxdist[v] + std::sqrt(c.rneighbordist2_unit[u * c.nunit + v])) val = 1;
      }
      neigh_unit[u * c.nunit + v] = val;
    }

  r.iexv2mp.clear();
  for (int imp = 0; imp < c.nmp; ++imp) {
    int iunit = c.imp2unit[imp];
    int jmp = imp + 1;
    while (jmp < c.nmp) {
      int junit = c.imp2unit[jmp];
      if (neigh_unit[iunit * c.nunit + junit] == 1) {
        double v21[3];
        for (int k = 0; k < 3; ++k) v21[k] = X[3 * jmp + k] - X[3 * imp + k];
        if (peri) pbneighbor(c, v21, nullptr);
        double dist2 = v21[0] * v21[0] + v21[1] * v21[1] + v21[2] * v21[2];
        if (dist2 < c.rneighbordist2_unit[iunit * c.nunit + junit]) {
          // neighbor_assign.F90:481-558
          int ok = 0;
          int ci = c.iclass_unit[iunit], cj = c.iclass_unit[junit];
          if (iunit == junit) {
            ok = 1;
            if (ci == TIS_CLASS_RNA) {
              if (jmp + 1 < imp + 1 + nsep_of(c, imp)) ok = 0;
            }
          } else if (ci == TIS_CLASS_RNA && cj == TIS_CLASS_RNA) ok = 1;
          else if ((ci == TIS_CLASS_RNA && cj == TIS_CLASS_ION) || (ci == TIS_CLASS_ION && cj == TIS_CLASS_RNA)) {
            ok = 1;
            // neighbor_assign.F90:524-537: no exv between a charged phosphate and an ion
            if (c.dt19) {
              const Label &L = c.lab[r.label - 1];
              int pb = (c.imp2type[imp] == TIS_MP_RNA_PHOS) ? imp : (c.imp2type[jmp] == TIS_MP_RNA_PHOS ? jmp : -1);
              if (pb >= 0 && c.lmp2charge[pb] >= 0 && std::fabs(qch(c, L, c.lmp2charge[pb])) > ZERO_JUDGE) ok = 0;
            }
          } else if ((ci == TIS_CLASS_ION && cj == TIS_CLASS_LIG) || (ci == TIS_CLASS_LIG && cj == TIS_CLASS_ION)) ok = 1;
          if (ok) {
            r.iexv2mp.push_back(imp + 1);
            r.iexv2mp.push_back(jmp + 1);
            r.iexv2mp.push_back(1);
          }
        }
      } else {
        jmp = c.lunit2mp[2 * junit + 1] - 1;   // jump to the last bead of junit
      }
      ++jmp;
    }
  }
  // neighbor_assign.F90:742-770
  size_t nexv = r.iexv2mp.size() / 3;
  for (size_t e = 0; e < nexv; ++e) {
    if (peri) {
      int imp = r.iexv2mp[3 * e] - 1, jmp = r.iexv2mp[3 * e + 1] - 1;
      double vx[3];
      for (int k = 0; k < 3; ++k) vx[k] = r.pxyz[3 * jmp + k] - r.pxyz[3 * imp + k];
      int im; pbneighbor(c, vx, &im);
      r.iexv2mp[3 * e + 2] = im;
    } else {
      r.iexv2mp[3 * e + 2] = 1;
    }
  }
}

// neighbor_list_ele.F90:59-210 (i_neigh_dynamic = 1, unit flags all set)
void neighbor_ele(orc_ctx &c, Rep &r) {
  r.iele2mp.clear(); r.coef_ele.clear();
  if (c.par.i_ele == TIS_ELE_NONE) return;
  const Label &L = c.lab[r.label - 1];
  double rneighbor2_ele;
  if (c.par.i_ele == TIS_ELE_DH)
    rneighbor2_ele = sq(c.par.neigh_margin + c.par.cutoff_ele * L.cdist);
  else
    rneighbor2_ele = sq(c.par.neigh_margin + c.par.cutoff_ele);
  const bool peri = c.par.i_periodic == 1;
  const double *X = peri ? r.pxyz.data() : r.xyz.data();
  for (int ic = 0; ic < c.ncharge - 1; ++ic) {
    if (std::fabs(qch(c, L, ic)) < ZERO_JUDGE) continue;
    int imp = c.icharge2mp[ic];
    for (int jc = ic + 1; jc < c.ncharge; ++jc) {
      if (std::fabs(qch(c, L, jc)) < ZERO_JUDGE) continue;
      int jmp = c.icharge2mp[jc];
      double v21[3];
      for (int k = 0; k < 3; ++k) v21[k] = X[3 * jmp + k] - X[3 * imp + k];
      int imirror = 1;
      if (peri) pbneighbor(c, v21, &imirror);
      double dist2 = v21[0] * v21[0] + v21[1] * v21[1] + v21[2] * v21[2];
      if (dist2 < rneighbor2_ele) {
        r.iele2mp.push_back(imp + 1);
        r.iele2mp.push_back(jmp + 1);
        r.iele2mp.push_back(peri ? imirror : 1);
        r.iele2mp.push_back((c.dt19 && is_mg_p(c, imp, jmp)) ? 1 : 0);   // neighbor_list_ele.F90:167-174
        r.coef_ele.push_back(qch(c, L, ic) * qch(c, L, jc) * L.coef);
      }
    }
  }
}

// neighbor_list_hb.F90:322-410 (the per-site lists are the static ones
// filtered by hb_status when the pruning reads them)
void neighbor_hb(orc_ctx &c, Rep &r) {
  r.ineigh2hb.clear();
  const bool peri = c.par.i_periodic == 1;
  for (int ihb = 0; ihb < c.nhb; ++ihb) {
    int a = c.hb2mp[6 * ihb] - 1, b = c.hb2mp[6 * ihb + 1] - 1;
    double v12[3];
    const double *X = peri ? r.pxyz.data() : r.xyz.data();
    for (int k = 0; k < 3; ++k) v12[k] = X[3 * a + k] - X[3 * b + k];
    if (peri) pbneighbor(c, v12, nullptr);
    double d1212 = dot3(v12, v12);
    if (d1212 < c.hb_neigh_dist2[ihb]) r.ineigh2hb.push_back(ihb + 1);
  }
}

// neighbor.F90:13-99
void neighbor(orc_ctx &c, Rep &r) {
  if (c.par.i_periodic == 1) util_periodic(c, r);
  neighbor_exv(c, r);
  neighbor_ele(c, r);
  neighbor_hb(c, r);
  r.nrebuild++;
  r.last_rebuild = r.istep;
}

// ------------------------------------------------------------ force terms
// force_bond.F90:41-56
void force_bond(const orc_ctx &c, const Rep &r, double *F) {
  for (int ibd = 0; ibd < c.nbd; ++ibd) {
    int i1 = c.ibd2mp[2 * ibd] - 1, i2 = c.ibd2mp[2 * ibd + 1] - 1;
    double v21[3];
    for (int k = 0; k < 3; ++k) v21[k] = r.xyz[3 * i2 + k] - r.xyz[3 * i1 + k];
    double dist = std::sqrt(v21[0] * v21[0] + v21[1] * v21[1] + v21[2] * v21[2]);
    double ddist = dist - c.bd_nat[ibd];
    double f = c.coef_bd[ibd] * (-2.0e0 * ddist / dist);
    for (int k = 0; k < 3; ++k) {
      double fk = f * v21[k];
      F[3 * i1 + k] = F[3 * i1 + k] - fk;
      F[3 * i2 + k] = F[3 * i2 + k] + fk;
    }
  }
}

// force_fene.F90 (loop body)
void force_fene(const orc_ctx &c, const Rep &r, double *F) {
  for (int i = 0; i < c.nfene; ++i) {
    int i1 = c.fene2mp[2 * i] - 1, i2 = c.fene2mp[2 * i + 1] - 1;
    double v21[3];
    for (int k = 0; k < 3; ++k) v21[k] = r.xyz[3 * i2 + k] - r.xyz[3 * i1 + k];
    double dist = norm2_3(v21);
    double ddist = dist - c.fene_nat[i];
    double ddist2 = ddist * ddist;
    double f = -c.coef_fene[i] * ddist / (1.0 - ddist2 / c.dist2_fene[i]) / dist;
    for (int k = 0; k < 3; ++k) {
      double fk = f * v21[k];
      F[3 * i1 + k] = F[3 * i1 + k] - fk;
      F[3 * i2 + k] = F[3 * i2 + k] + fk;
    }
  }
}

// force_bangle.F90:103-147 (default build, no _HTN_CONSISTENT)
void force_bangle(const orc_ctx &c, const Rep &r, double *F) {
  for (int iba = 0; iba < c.nba; ++iba) {
    if (c.coef_ba[iba] < ZERO_JUDGE) continue;
    int i1 = c.iba2mp[3 * iba] - 1, i2 = c.iba2mp[3 * iba + 1] - 1, i3 = c.iba2mp[3 * iba + 2] - 1;
    double v21[3], v32[3];
    for (int k = 0; k < 3; ++k) {
      v21[k] = r.xyz[3 * i2 + k] - r.xyz[3 * i1 + k];
      v32[k] = r.xyz[3 * i3 + k] - r.xyz[3 * i2 + k];
    }
    double c11 = v21[0] * v21[0] + v21[1] * v21[1] + v21[2] * v21[2];
    double c22 = v32[0] * v32[0] + v32[1] * v32[1] + v32[2] * v32[2];
    double c21 = v32[0] * v21[0] + v32[1] * v21[1] + v32[2] * v21[2];
    double co = -c21 / std::sqrt(c11 * c22);
    if (co > 1.0e0) co = 1.0e0;
    else if (co < -1.0e0) co = -1.0e0;
    double dba = std::acos(co) - c.ba_nat[iba];
    double t3 = c11 * c22 - c21 * c21;
    if (t3 <= 1.0e0) t3 = 1.0e0;
    double f = 2.0e0 * c.coef_ba[iba] * dba / std::sqrt(t3);
    for (int k = 0; k < 3; ++k) {
      double f21 = f * (v21[k] * (c21 / c11) - v32[k]);
      double f32 = f * (v32[k] * (c21 / c22) - v21[k]);
      F[3 * i1 + k] = F[3 * i1 + k] - f21;
      F[3 * i2 + k] = F[3 * i2 + k] + f21 - f32;
      F[3 * i3 + k] = F[3 * i3 + k] + f32;
    }
  }
}

inline void cross(const double *a, const double *b, double *o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
inline double wrap_pi(double d) {
  if (d > F_PI) d = d - F_2PI;
  else if (d < -F_PI) d = d + F_2PI;
  return d;
}

// force_dtrna_stack.F90:54-165
void force_dtrna_stack(const orc_ctx &c, const Rep &r, double *F) {
  const Label &L = c.lab[r.label - 1];
  for (int ist = 0; ist < c.nst; ++ist) {
    if (!r.st_status[ist]) continue;
    const int *m7 = &c.st2mp[7 * ist];
    auto X = [&](int k, int d) { return r.xyz[3 * (m7[k] - 1) + d]; };
    double v21[3], v34[3], v54[3], v56[3], v76[3];
    for (int d = 0; d < 3; ++d) {
      v21[d] = X(1, d) - X(0, d);
      v34[d] = X(2, d) - X(3, d);
      v54[d] = X(4, d) - X(3, d);
      v56[d] = X(4, d) - X(5, d);
      v76[d] = X(6, d) - X(5, d);
    }
    double k1 = c.st_coef[3 * ist], k2 = c.st_coef[3 * ist + 1], k3 = c.st_coef[3 * ist + 2];
    double ediv = 1.0e0;
    double fr[7][3] = {{0}};
    double dist = norm2_3(v21);
    double ddist = dist - c.st_nat[3 * ist];
    ediv = ediv + k1 * ddist * ddist;
    double fi[3], fl[3];
    for (int d = 0; d < 3; ++d) {
      fi[d] = 2.0e0 * k1 * ddist / dist * v21[d];
      fr[0][d] = -fi[d];
      fr[1][d] = +fi[d];
    }
    double m[3], n[3];
    cross(v34, v54, m);
    cross(v54, v56, n);
    double dmm = dot3(m, m), dnn = dot3(n, n);
    double d5454 = dot3(v54, v54);
    double abs54 = std::sqrt(d5454);
    double d5654 = dot3(v56, v54);
    double d3454over5454 = dot3(v34, v54) / d5454;
    double d5654over5454 = d5654 / d5454;
    double dih = std::atan2(dot3(v34, n) * std::sqrt(d5454), dot3(m, n));
    double dd = wrap_pi(dih - c.st_nat[3 * ist + 1]);
    ediv = ediv + k2 * dd * dd;
    for (int d = 0; d < 3; ++d) {
      fi[d] = +2.0e0 * k2 * dd * abs54 / dmm * m[d];
      fl[d] = -2.0e0 * k2 * dd * abs54 / dnn * n[d];
    }
    for (int d = 0; d < 3; ++d) {
      fr[2][d] = fi[d];
      fr[3][d] = (-1.0e0 + d3454over5454) * fi[d] - (d5654over5454) * fl[d];
      fr[4][d] = (-1.0e0 + d5654over5454) * fl[d] - (d3454over5454) * fi[d];
      fr[5][d] = fl[d];
    }
    cross(v76, v56, m);
    for (int d = 0; d < 3; ++d) n[d] = -n[d];
    dmm = dot3(m, m);
    double d5656 = dot3(v56, v56);
    double abs56 = std::sqrt(d5656);
    double d7656over5656 = dot3(v76, v56) / d5656;
    double d5456over5656 = d5654 / d5656;
    dih = std::atan2(dot3(v76, n) * std::sqrt(d5656), dot3(m, n));
    dd = wrap_pi(dih - c.st_nat[3 * ist + 2]);
    ediv = ediv + k3 * dd * dd;
    for (int d = 0; d < 3; ++d) {
      fi[d] = +2.0e0 * k3 * dd * abs56 / dmm * m[d];
      fl[d] = -2.0e0 * k3 * dd * abs56 / dnn * n[d];
    }
    for (int d = 0; d < 3; ++d) {
      fr[6][d] = fr[6][d] + fi[d];
      fr[5][d] = fr[5][d] + (-1.0e0 + d7656over5656) * fi[d] - (d5456over5656) * fl[d];
      fr[4][d] = fr[4][d] - (d7656over5656) * fi[d] + (-1.0e0 + d5456over5656) * fl[d];
      fr[3][d] = fr[3][d] + fl[d];
    }
    double pre = L.st_u0[ist] / (ediv * ediv);
    for (int k = 0; k < 7; ++k)
      for (int d = 0; d < 3; ++d) fr[k][d] = pre * fr[k][d];
    for (int k = 0; k < 7; ++k)
      for (int d = 0; d < 3; ++d) F[3 * (m7[k] - 1) + d] = F[3 * (m7[k] - 1) + d] + fr[k][d];
  }
}

// force_dtrna_stack_nlocal.F90:60-263 (forces) and energy_dtrna_stack_nlocal.F90
// (energy, U0 / ediv): sets st_status of the secondary stacks that a
// tertiary stack within 10 A of its native distance excludes.  F may be null
// (energy only); returns the tertiary stacking energy.
double dtrna_stack_nlocal(const orc_ctx &c, Rep &r, double *F) {
  const bool peri = c.par.i_periodic == 1;
  const double *X = peri ? r.pxyz.data() : r.xyz.data();
  r.st_status.assign(c.nst, 1);
  double etot = 0.0;
  for (int ist = 0; ist < c.ntst; ++ist) {
    const int *m = &c.tst2mp[6 * ist];
    const double *nat = &c.tst_nat[6 * ist];
    const double *cf = &c.tst_coef[7 * ist];
    auto dv = [&](int p, int q, double *v) {
      for (int d = 0; d < 3; ++d) v[d] = X[3 * (m[p] - 1) + d] - X[3 * (m[q] - 1) + d];
      if (peri) { int im; pbneighbor(c, v, &im); }
    };
    double v12[3], v13[3], v53[3], v42[3], v46[3];
    dv(0, 1, v12);
    const double d1212 = dot3(v12, v12);
    const double a12 = std::sqrt(d1212);
    double d = a12 - nat[0];
    if (d < 10.0) {
      for (int sd = 0; sd < 2; ++sd)
        if (c.tst_excl[2 * ist + sd]) r.st_status[c.tst2st[2 * ist + sd]] = 0;
    }
    double ediv = 1.0e0;
    double fr[6][3] = {{0}};
    dv(0, 2, v13); dv(4, 2, v53); dv(3, 1, v42); dv(3, 5, v46);
    const double d1313 = dot3(v13, v13), d4242 = dot3(v42, v42);
    const double a13 = std::sqrt(d1313), a42 = std::sqrt(d4242);
    const double d1213 = dot3(v13, v12), d1242 = dot3(v12, v42), d4246 = dot3(v42, v46), d1353 = dot3(v13, v53);
    const double d1213over1212 = d1213 / d1212, d1213over1313 = d1213 / d1313;
    const double d1242over1212 = d1242 / d1212, d4246over4242 = d4246 / d4242;
    const double d1242over4242 = d1242 / d4242, d1353over1313 = d1353 / d1313;
    double fi[3], fk[3], fl[3];
    // distance 1=2
    ediv = ediv + cf[1] * d * d;
    for (int q = 0; q < 3; ++q) {
      fi[q] = 2.0e0 * cf[1] * d * v12[q] / a12;
      fr[0][q] = +fi[q];
      fr[1][q] = -fi[q];
    }
    // angle 3-1=2
    double cos_theta = d1213 / (a13 * a12);
    d = std::acos(cos_theta) - nat[1];
    double pre = 2.0e0 * cf[2] * d / std::sqrt(d1313 * d1212 - d1213 * d1213);
    for (int q = 0; q < 3; ++q) {
      fi[q] = pre * (v12[q] - (d1213over1313 * v13[q]));
      fk[q] = pre * (v13[q] - (d1213over1212 * v12[q]));
      fr[2][q] = fr[2][q] + fi[q];
      fr[1][q] = fr[1][q] + fk[q];
      fr[0][q] = fr[0][q] - fi[q] - fk[q];
    }
    ediv = ediv + cf[2] * d * d;
    // angle 1=2-4
    cos_theta = d1242 / (a12 * a42);
    d = std::acos(cos_theta) - nat[2];
    pre = 2.0e0 * cf[3] * d / std::sqrt(d1212 * d4242 - d1242 * d1242);
    for (int q = 0; q < 3; ++q) {
      fi[q] = -pre * (v42[q] - (d1242over1212 * v12[q]));
      fk[q] = -pre * (v12[q] - (d1242over4242 * v42[q]));
      fr[0][q] = fr[0][q] + fi[q];
      fr[3][q] = fr[3][q] + fk[q];
      fr[1][q] = fr[1][q] - fi[q] - fk[q];
    }
    ediv = ediv + cf[3] * d * d;
    // dihedral 4-2=1=3
    double c4212[3], c1213[3];
    cross(v42, v12, c4212);
    cross(v12, v13, c1213);
    const double c4212_abs2 = dot3(c4212, c4212), c1213_abs2 = dot3(c1213, c1213);
    double dih = std::atan2(dot3(v42, c1213) * std::sqrt(d1212), dot3(c4212, c1213));
    d = wrap_pi(dih - nat[3]);
    ediv = ediv + cf[4] * d * d;
    pre = 2.0e0 * cf[4] * d * a12;
    for (int q = 0; q < 3; ++q) {
      fi[q] = +pre / c4212_abs2 * c4212[q];
      fl[q] = -pre / c1213_abs2 * c1213[q];
    }
    for (int q = 0; q < 3; ++q) {
      fr[3][q] = fr[3][q] + fi[q];
      fr[1][q] = fr[1][q] + (-1.0e0 + d1242over1212) * fi[q] - (d1213over1212) * fl[q];
      fr[0][q] = fr[0][q] + (-1.0e0 + d1213over1212) * fl[q] - (d1242over1212) * fi[q];
      fr[2][q] = fr[2][q] + fl[q];
    }
    // dihedral 5-3-1=2
    double mm[3], nn[3];
    cross(v53, v13, mm);
    for (int q = 0; q < 3; ++q) nn[q] = -c1213[q];
    double dmm = dot3(mm, mm), dnn = c1213_abs2;
    dih = std::atan2(dot3(v53, nn) * a13, dot3(mm, nn));
    d = wrap_pi(dih - nat[4]);
    ediv = ediv + cf[5] * d * d;
    pre = 2.0e0 * cf[5] * d * a13;
    for (int q = 0; q < 3; ++q) {
      fi[q] = +pre / dmm * mm[q];
      fl[q] = -pre / dnn * nn[q];
    }
    for (int q = 0; q < 3; ++q) {
      fr[4][q] = fr[4][q] + fi[q];
      fr[2][q] = fr[2][q] + (-1.0e0 + d1353over1313) * fi[q] - (d1213over1313) * fl[q];
      fr[0][q] = fr[0][q] + (-1.0e0 + d1213over1313) * fl[q] - (d1353over1313) * fi[q];
      fr[1][q] = fr[1][q] + fl[q];
    }
    // dihedral 1=2-4-6
    for (int q = 0; q < 3; ++q) mm[q] = -c4212[q];
    cross(v42, v46, nn);
    dmm = c4212_abs2;
    dnn = dot3(nn, nn);
    dih = std::atan2(dot3(v12, nn) * a42, dot3(mm, nn));
    d = wrap_pi(dih - nat[5]);
    ediv = ediv + cf[6] * d * d;
    pre = 2.0e0 * cf[6] * d * a42;
    for (int q = 0; q < 3; ++q) {
      fi[q] = +pre / dmm * mm[q];
      fl[q] = -pre / dnn * nn[q];
    }
    for (int q = 0; q < 3; ++q) {
      fr[0][q] = fr[0][q] + fi[q];
      fr[1][q] = fr[1][q] + (-1.0e0 + d1242over4242) * fi[q] - (d4246over4242) * fl[q];
      fr[3][q] = fr[3][q] + (-1.0e0 + d4246over4242) * fl[q] - (d1242over4242) * fi[q];
      fr[5][q] = fr[5][q] + fl[q];
    }
    etot += cf[0] / ediv;
    if (F) {
      for (int k = 0; k < 6; ++k)
        for (int q = 0; q < 3; ++q) F[3 * (m[k] - 1) + q] = F[3 * (m[k] - 1) + q] + fr[k][q] * cf[0] / (ediv * ediv);
    }
  }
  return etot;
}

double draw_uniform(Rep &r) {
  if (r.upos < r.unif.size()) return r.unif[r.upos++];
  r.unif_exhausted = true;
  return 0.5;
}

// force_dtrna_hbond15.F90:71-353: per-hbond force and energy into for_hb,
// ene_hb and hb_status; counts hbsite_excess.
void hbond15_terms(orc_ctx &c, Rep &r) {
  r.hb_status.assign(c.nhb, 0);
  r.hbsite_excess.assign(c.nhbsite, 0);
  r.ene_hb.assign(c.nhb, 0.0);
  r.for_hb.assign(18 * (size_t)c.nhb, 0.0);
  const bool peri = c.par.i_periodic == 1;
  for (size_t ineigh = 0; ineigh < r.ineigh2hb.size(); ++ineigh) {
    int ihb = r.ineigh2hb[ineigh] - 1;
    const int *m6 = &c.hb2mp[6 * ihb];
    const double *nat = &c.hb_nat[6 * ihb];
    const double *cf = &c.hb_coef[7 * ihb];   // cf[0] = U0
    double *fo = &r.for_hb[18 * (size_t)ihb];   // fo[3*k + d]
    auto Xv = [&](int k, int d) { return r.xyz[3 * (m6[k] - 1) + d]; };
    auto Pv = [&](int k, int d) { return r.pxyz[3 * (m6[k] - 1) + d]; };
    double v12[3];
    if (!peri) for (int d = 0; d < 3; ++d) v12[d] = Xv(0, d) - Xv(1, d);
    else { for (int d = 0; d < 3; ++d) v12[d] = Pv(0, d) - Pv(1, d); pbneighbor(c, v12, nullptr); }
    double d1212 = dot3(v12, v12);
    double a12 = std::sqrt(d1212);
    double d = a12 - nat[0];
    if (std::fabs(d) > c.par.hb_cutoff_dist) continue;
    r.hb_status[ihb] = 1;
    for (int i = 0; i < 3; ++i) {
      int s = c.hb2site[6 * ihb + i];
      if (s > 0) r.hbsite_excess[s - 1] += 1;
    }
    for (int i = 0; i < 3; ++i) {
      int s = c.hb2site[6 * ihb + 3 + i];
      if (s > 0) r.hbsite_excess[s - 1] += 1;
    }
    double ex = -cf[1] * d * d;
    double fi[3], fk[3], fl[3];
    for (int k = 0; k < 3; ++k) {
      fi[k] = (2.0e0 * cf[1] * d / a12) * v12[k];
      fo[0 * 3 + k] = +fi[k];
      fo[1 * 3 + k] = -fi[k];
    }
    double v13[3], v53[3], v42[3], v46[3];
    for (int k = 0; k < 3; ++k) {
      v13[k] = Xv(0, k) - Xv(2, k);
      v53[k] = Xv(4, k) - Xv(2, k);
      v42[k] = Xv(3, k) - Xv(1, k);
      v46[k] = Xv(3, k) - Xv(5, k);
    }
    if (peri) {
      pbneighbor(c, v13, nullptr); pbneighbor(c, v53, nullptr);
      pbneighbor(c, v42, nullptr); pbneighbor(c, v46, nullptr);
    }
    double d1313 = dot3(v13, v13), d4242 = dot3(v42, v42);
    double a13 = std::sqrt(d1313), a42 = std::sqrt(d4242);
    double d1213 = dot3(v13, v12), d1242 = dot3(v12, v42);
    double d4246 = dot3(v42, v46), d1353 = dot3(v13, v53);
    double d1213over1212 = d1213 / d1212, d1213over1313 = d1213 / d1313;
    double d1242over1212 = d1242 / d1212, d4246over4242 = d4246 / d4242;
    double d1242over4242 = d1242 / d4242, d1353over1313 = d1353 / d1313;

    // angle 3-1=2 (lines 197-209)
    double cos312 = d1213 / (a13 * a12);
    if (std::fabs(cos312) > MAX_ANG_ABSCOS_HBOND15)
      d1213 = std::copysign(a12 * a13 * MAX_ANG_ABSCOS_HBOND15, cos312);
    d = std::acos(cos312) - nat[1];
    double pre = 2.0e0 * cf[2] * d / std::sqrt(d1313 * d1212 - d1213 * d1213);
    for (int k = 0; k < 3; ++k) {
      fi[k] = pre * (v12[k] - (d1213over1313 * v13[k]));
      fk[k] = pre * (v13[k] - (d1213over1212 * v12[k]));
      fo[2 * 3 + k] = fo[2 * 3 + k] + fi[k];
      fo[1 * 3 + k] = fo[1 * 3 + k] + fk[k];
      fo[0 * 3 + k] = fo[0 * 3 + k] - fi[k] - fk[k];
    }
    ex = ex - cf[2] * d * d;

    // angle 1=2-4 (lines 227-239)
    double cos124 = d1242 / (a12 * a42);
    if (std::fabs(cos124) > MAX_ANG_ABSCOS_HBOND15)
      d1242 = std::copysign(a12 * a42 * MAX_ANG_ABSCOS_HBOND15, cos124);
    d = std::acos(cos124) - nat[2];
    pre = 2.0e0 * cf[3] * d / std::sqrt(d1212 * d4242 - d1242 * d1242);
    for (int k = 0; k < 3; ++k) {
      fi[k] = -pre * (v42[k] - (d1242over1212 * v12[k]));
      fk[k] = -pre * (v12[k] - (d1242over4242 * v42[k]));
      fo[0 * 3 + k] = fo[0 * 3 + k] + fi[k];
      fo[3 * 3 + k] = fo[3 * 3 + k] + fk[k];
      fo[1 * 3 + k] = fo[1 * 3 + k] - fi[k] - fk[k];
    }
    ex = ex - cf[3] * d * d;

    // dihedral 4-2=1=3 (lines 243-278)
    double c4212[3], c1213[3];
    cross(v42, v12, c4212);
    cross(v12, v13, c1213);
    double c4212_abs2 = dot3(c4212, c4212), c1213_abs2 = dot3(c1213, c1213);
    if (std::fabs(cos124) > MAX_DIH_ABSCOS_HBOND15)
      c4212_abs2 = d4242 * d1212 * (1.0 - MAX_DIH_ABSCOS_HBOND15 * MAX_DIH_ABSCOS_HBOND15);
    if (std::fabs(cos312) > MAX_DIH_ABSCOS_HBOND15)
      c1213_abs2 = d1212 * d1313 * (1.0 - MAX_DIH_ABSCOS_HBOND15 * MAX_DIH_ABSCOS_HBOND15);
    double dih = std::atan2(dot3(v42, c1213) * a12, dot3(c4212, c1213));
    d = wrap_pi(dih - nat[3]);
    ex = ex - cf[4] * d * d;
    pre = 2.0e0 * cf[4] * d * a12;
    for (int k = 0; k < 3; ++k) {
      fi[k] = +pre / c4212_abs2 * c4212[k];
      fl[k] = -pre / c1213_abs2 * c1213[k];
    }
    for (int k = 0; k < 3; ++k) {
      fo[3 * 3 + k] = fo[3 * 3 + k] + fi[k];
      fo[1 * 3 + k] = fo[1 * 3 + k] + (-1.0e0 + d1242over1212) * fi[k] - (d1213over1212) * fl[k];
      fo[0 * 3 + k] = fo[0 * 3 + k] + (-1.0e0 + d1213over1212) * fl[k] - (d1242over1212) * fi[k];
      fo[2 * 3 + k] = fo[2 * 3 + k] + fl[k];
    }

    // dihedral 5-3-1=2 (lines 282-311)
    double c5313[3], n[3];
    cross(v53, v13, c5313);
    for (int k = 0; k < 3; ++k) n[k] = -c1213[k];
    double c5313_abs2 = dot3(c5313, c5313);
    double cos531 = d1353 / (a13 * norm2_3(v53));
    if (std::fabs(cos531) > MAX_DIH_ABSCOS_HBOND15)
      c5313_abs2 = dot3(v53, v53) * d1313 * (1.0 - MAX_DIH_ABSCOS_HBOND15 * MAX_DIH_ABSCOS_HBOND15);
    dih = std::atan2(dot3(v53, n) * a13, dot3(c5313, n));
    d = wrap_pi(dih - nat[4]);
    ex = ex - cf[5] * d * d;
    pre = 2.0e0 * cf[5] * d * a13;
    for (int k = 0; k < 3; ++k) {
      fi[k] = +pre / c5313_abs2 * c5313[k];
      fl[k] = -pre / c1213_abs2 * n[k];
    }
    for (int k = 0; k < 3; ++k) {
      fo[4 * 3 + k] = fo[4 * 3 + k] + fi[k];
      fo[2 * 3 + k] = fo[2 * 3 + k] + (-1.0e0 + d1353over1313) * fi[k] - (d1213over1313) * fl[k];
      fo[0 * 3 + k] = fo[0 * 3 + k] + (-1.0e0 + d1213over1313) * fl[k] - (d1353over1313) * fi[k];
      fo[1 * 3 + k] = fo[1 * 3 + k] + fl[k];
    }

    // dihedral 1=2-4-6 (lines 315-344)
    for (int k = 0; k < 3; ++k) n[k] = -c4212[k];
    double c4246[3];
    cross(v42, v46, c4246);
    double c4246_abs2 = dot3(c4246, c4246);
    double cos246 = d4246 / (a42 * norm2_3(v46));
    if (std::fabs(cos246) > MAX_DIH_ABSCOS_HBOND15)
      c4246_abs2 = dot3(v46, v46) * d4242 * (1.0 - MAX_DIH_ABSCOS_HBOND15 * MAX_DIH_ABSCOS_HBOND15);
    dih = std::atan2(dot3(v12, c4246) * a42, dot3(n, c4246));
    d = wrap_pi(dih - nat[5]);
    ex = ex - cf[6] * d * d;
    pre = 2.0e0 * cf[6] * d * a42;
    for (int k = 0; k < 3; ++k) {
      fi[k] = +pre / c4212_abs2 * n[k];
      fl[k] = -pre / c4246_abs2 * c4246[k];
    }
    for (int k = 0; k < 3; ++k) {
      fo[0 * 3 + k] = fo[0 * 3 + k] + fi[k];
      fo[1 * 3 + k] = fo[1 * 3 + k] + (-1.0e0 + d1242over4242) * fi[k] - (d4246over4242) * fl[k];
      fo[3 * 3 + k] = fo[3 * 3 + k] + (-1.0e0 + d4246over4242) * fl[k] - (d1242over4242) * fi[k];
      fo[5 * 3 + k] = fo[5 * 3 + k] + fl[k];
    }
    double ene = cf[0] * std::exp(ex);
    r.ene_hb[ihb] = ene;
    for (int k = 0; k < 18; ++k) fo[k] = ene * fo[k];
  }
}

// force_dtrna_hbond15.F90:373-509: valence-excess pruning, drawing from the
// replica's uniform stream in the reference's order.
void hbond15_prune(orc_ctx &c, Rep &r, bool zero_energy) {
  for (int s = 0; s < c.nhbsite; ++s) r.hbsite_excess[s] -= c.nvalence[s];
  std::vector<int> excess_list;
  auto rebuild_list = [&]() {
    excess_list.clear();
    for (int s = 0; s < c.nhbsite; ++s)
      if (r.hbsite_excess[s] > 0) excess_list.push_back(s + 1);
  };
  rebuild_list();
  std::vector<int> seq;
  while (!excess_list.empty()) {
    int nex = (int)excess_list.size();
    double rnd = draw_uniform(r);   // genrand_double4: (0,1]
    int pick = (int)std::ceil(rnd * nex);
    if (pick < 1) pick = 1;
    if (pick > nex) pick = nex;
    int site = excess_list[pick - 1];
    seq.clear();
    for (int ihb : c.hb_at_site[site - 1])
      if (r.hb_status[ihb - 1]) seq.push_back(ihb);
    int nseq = (int)seq.size();
    for (int i = 0; i < nseq; ++i) {
      rnd = draw_uniform(r);        // genrand_double1: [0,1]
      int isw = (int)std::ceil(rnd * nseq);
      if (isw < 1) isw = 1;         // the reference indexes hb_seq(0) when rnd == 0
      std::swap(seq[i], seq[isw - 1]);
    }
    int idel = seq.empty() ? 0 : seq[0];
    for (int i = 1; i < nseq; ++i) {
      int jhb = seq[i];
      double ratio = std::exp((r.ene_hb[jhb - 1] - r.ene_hb[idel - 1]) * c.beta_hbond15);
      rnd = draw_uniform(r);
      if (rnd < ratio) idel = jhb;
    }
    if (idel == 0) break;   // no active hbond at an excess site: cannot happen for consistent tables
    r.hb_status[idel - 1] = 0;
    if (zero_energy) r.ene_hb[idel - 1] = 0.0;
    for (int i = 0; i < 3; ++i) {
      int s = c.hb2site[6 * (idel - 1) + i];
      if (s > 0 && r.hbsite_excess[s - 1] > 0) r.hbsite_excess[s - 1] -= 1;
      s = c.hb2site[6 * (idel - 1) + 3 + i];
      if (s > 0 && r.hbsite_excess[s - 1] > 0) r.hbsite_excess[s - 1] -= 1;
    }
    rebuild_list();
  }
}

void force_dtrna_hbond15(orc_ctx &c, Rep &r, double *F) {
  hbond15_terms(c, r);
  hbond15_prune(c, r, true);
  for (size_t ineigh = 0; ineigh < r.ineigh2hb.size(); ++ineigh) {
    int ihb = r.ineigh2hb[ineigh] - 1;
    if (!r.hb_status[ihb]) continue;
    const double *fo = &r.for_hb[18 * (size_t)ihb];
    for (int k = 0; k < 6; ++k) {
      int m = c.hb2mp[6 * ihb + k] - 1;
      for (int d = 0; d < 3; ++d) F[3 * m + d] = F[3 * m + d] + fo[3 * k + d];
    }
  }
}

// force_exv_dt15.F90:60-78
double exv_dij(const orc_ctx &c, int i1, int i2) {
  int t1 = c.imp2type[i1], t2 = c.imp2type[i2];
  if (c.dt19) {
    if (t1 == TIS_MP_RNA_BASE && t2 == TIS_MP_RNA_BASE) return c.par.exv_dist;
    return c.exv_radius[i1] + c.exv_radius[i2];
  }
  if (t1 == TIS_MP_RNA_PHOS && t2 == TIS_MP_RNA_SUGAR) return c.par.exv_dist_PS;
  if (t1 == TIS_MP_RNA_SUGAR && t2 == TIS_MP_RNA_PHOS) return c.par.exv_dist_PS;
  if (c.iclass_mp[i1] == TIS_CLASS_RNA && c.iclass_mp[i2] == TIS_CLASS_RNA) return c.par.exv_dist;
  return c.exv_radius[i1] + c.exv_radius[i2];
}

void force_exv_dt15(const orc_ctx &c, Rep &r, double *F) {
  double a = c.par.exv_adjust, a2 = a * a;
  size_t nexv = r.iexv2mp.size() / 3;
  for (size_t e = 0; e < nexv; ++e) {
    int i1 = r.iexv2mp[3 * e] - 1, i2 = r.iexv2mp[3 * e + 1] - 1, im = r.iexv2mp[3 * e + 2] - 1;
    double dij = exv_dij(c, i1, i2);
    double v21[3];
    for (int k = 0; k < 3; ++k) v21[k] = r.pxyz[3 * i2 + k] - r.pxyz[3 * i1 + k] + c.d_mirror[im][k];
    double dist = norm2_3(v21);
    if (dist > dij) continue;
    double coef = c.exv_epsilon[i1] * c.exv_epsilon[i2];
    double dr = dist + a - dij;
    double dr2 = dr * dr;
    double ro2 = a2 / dr2;
    double ro4 = ro2 * ro2;
    double ro8 = ro4 * ro4;
    double ro14 = ro2 * ro4 * ro8;
    double dv = std::fabs(12.0e0 * coef * (ro14 - ro8) * dr / a2 / dist);
    if (dv > DE_MAX) { dv = DE_MAX; r.nclamp++; }
    for (int k = 0; k < 3; ++k) {
      double fk = dv * v21[k];
      F[3 * i2 + k] = F[3 * i2 + k] + fk;
      F[3 * i1 + k] = F[3 * i1 + k] - fk;
    }
  }
}

// force_ele_DH.F90:42-117; Mg-P pairs of the DT19 model within pmf_rmax
// take the table force (:87-97)
void force_ele_DH(const orc_ctx &c, Rep &r, double *F) {
  const Label &L = c.lab[r.label - 1];
  double cutoff2 = sq(c.par.cutoff_ele * L.cdist);
  double rcdist = 1.0e0 / L.cdist;
  size_t nele = r.coef_ele.size();
  for (size_t e = 0; e < nele; ++e) {
    int i1 = r.iele2mp[4 * e] - 1, i2 = r.iele2mp[4 * e + 1] - 1, im = r.iele2mp[4 * e + 2] - 1;
    double v21[3];
    for (int k = 0; k < 3; ++k) v21[k] = r.pxyz[3 * i2 + k] - r.pxyz[3 * i1 + k] + c.d_mirror[im][k];
    double dist2 = dot3(v21, v21);
    if (dist2 > cutoff2) continue;
    double dist1 = std::sqrt(dist2);
    double rdist1 = 1.0 / dist1;
    double dv;
    if (r.iele2mp[4 * e + 3] > 0 && !L.pmf_f.empty() && dist1 <= c.par.pmf_rmax) {
      dv = rdist1 * L.pmf_f[pmf_bin(c, r, dist1)];
    } else {
      // coef_ele(iele) = coef_charge(i) * coef_charge(j) * inele%coef(grep), kept
      // current for the replica's temperature by simu_para2.F90
      double ce = qch(c, L, c.lmp2charge[i1]) * qch(c, L, c.lmp2charge[i2]) * L.coef;
      dv = ce * rdist1 * rdist1 * (rdist1 + rcdist) * std::exp(-dist1 * rcdist);
    }
    if (dv > DE_MAX) { dv = DE_MAX; r.nclamp++; }
    for (int k = 0; k < 3; ++k) {
      double fk = dv * v21[k];
      F[3 * i1 + k] = F[3 * i1 + k] - fk;
      F[3 * i2 + k] = F[3 * i2 + k] + fk;
    }
  }
}

// force_ele_coulomb.F90:55-82: coef_ele / r^3 along v21 inside the cutoff
// (A), no DE_MAX clamp
void force_ele_coulomb(const orc_ctx &c, Rep &r, double *F) {
  const Label &L = c.lab[r.label - 1];
  double cutoff2 = sq(c.par.cutoff_ele);
  size_t nele = r.coef_ele.size();
  for (size_t e = 0; e < nele; ++e) {
    int i1 = r.iele2mp[4 * e] - 1, i2 = r.iele2mp[4 * e + 1] - 1, im = r.iele2mp[4 * e + 2] - 1;
    double v21[3];
    for (int k = 0; k < 3; ++k) v21[k] = r.pxyz[3 * i2 + k] - r.pxyz[3 * i1 + k] + c.d_mirror[im][k];
    double dist2 = dot3(v21, v21);
    if (dist2 > cutoff2) continue;
    double dist1 = std::sqrt(dist2);
    double ce = qch(c, L, c.lmp2charge[i1]) * qch(c, L, c.lmp2charge[i2]) * L.coef;
    double dv_dr = ce / (dist1 * dist2);
    for (int k = 0; k < 3; ++k) {
      double fk = dv_dr * v21[k];
      F[3 * i1 + k] = F[3 * i1 + k] - fk;
      F[3 * i2 + k] = F[3 * i2 + k] + fk;
    }
  }
}

// force_ele_coulomb_ewld.F90:215-313
void force_ele_ewald(const orc_ctx &c, Rep &r, double *F) {
  const Label &L = c.lab[r.label - 1];
  double cutoff2 = sq(c.par.cutoff_ele);
  double alpha2 = sq(c.par.ewld_alpha);
  double beta = 2.0 * c.par.ewld_alpha / std::sqrt(F_PI);
  std::vector<double> qc(c.ncharge), qs(c.ncharge);
  for (int ig = 0; ig < c.ewld_f_n; ++ig) {
    const double *k = &c.ewld_f_rlv[3 * ig];
    for (int ic = 0; ic < c.ncharge; ++ic) {
      int imp = c.icharge2mp[ic];
      double dp = dot3(k, &r.pxyz[3 * imp]);
      double q1 = qch(c, L, ic);
      qc[ic] = q1 * std::cos(dp);
      qs[ic] = q1 * std::sin(dp);
    }
    double scos = 0.0, ssin = 0.0;
    for (int ic = 0; ic < c.ncharge; ++ic) scos += qc[ic];
    for (int ic = 0; ic < c.ncharge; ++ic) ssin += qs[ic];
    for (int ic = 0; ic < c.ncharge; ++ic) {
      int imp = c.icharge2mp[ic];
      double dv = L.coef * 2.0 * c.ewld_f_coef[ig] * (qs[ic] * scos - qc[ic] * ssin);
      for (int d = 0; d < 3; ++d) F[3 * imp + d] = F[3 * imp + d] + dv * k[d];
    }
  }
  size_t nele = r.coef_ele.size();
  for (size_t e = 0; e < nele; ++e) {
    int i1 = r.iele2mp[4 * e] - 1, i2 = r.iele2mp[4 * e + 1] - 1, im = r.iele2mp[4 * e + 2] - 1;
    double v21[3];
    for (int k = 0; k < 3; ++k) v21[k] = r.pxyz[3 * i2 + k] - r.pxyz[3 * i1 + k] + c.d_mirror[im][k];
    double dist2 = dot3(v21, v21);
    if (dist2 > cutoff2) continue;
    double dist1 = std::sqrt(dist2);
    double ce = qch(c, L, c.lmp2charge[i1]) * qch(c, L, c.lmp2charge[i2]) * L.coef;
    double dv = ce * (std::erfc(c.par.ewld_alpha * dist1) / dist1 + beta * std::exp(-alpha2 * dist2)) / dist2;
    for (int k = 0; k < 3; ++k) {
      double fk = dv * v21[k];
      F[3 * i1 + k] = F[3 * i1 + k] - fk;
      F[3 * i2 + k] = F[3 * i2 + k] + fk;
    }
  }
}

// force_wca.F90 (loop body); rcut_off2 = 1 / wca_coef_cutoff**2
void force_wca(const orc_ctx &c, Rep &r, double *F) {
  double rcut_off2 = 1.0 / sq(c.par.wca_coef_cutoff);
  const bool peri = c.par.i_periodic == 1;
  for (int i = 0; i < c.nwca; ++i) {
    int i1 = c.wca2mp[2 * i] - 1, i2 = c.wca2mp[2 * i + 1] - 1;
    double v21[3];
    if (!peri) for (int k = 0; k < 3; ++k) v21[k] = r.xyz[3 * i2 + k] - r.xyz[3 * i1 + k];
    else { for (int k = 0; k < 3; ++k) v21[k] = r.pxyz[3 * i2 + k] - r.pxyz[3 * i1 + k]; pbneighbor(c, v21, nullptr); }
    double dist2 = dot3(v21, v21);
    double nat2 = c.wca_nat[i] * c.wca_nat[i];
    double ro2 = nat2 / dist2;
    if (ro2 < rcut_off2) continue;
    double ro14 = std::pow(ro2, 7), ro8 = std::pow(ro2, 4);
    double coef = (ro2 > 1.0e0) ? c.coef_wca[i] : c.coef_wca[c.nwca + i];
    double dw = 12.0e0 * coef / nat2 * (ro14 - ro8);
    if (dw > DE_MAX) { dw = DE_MAX; r.nclamp++; }
    for (int k = 0; k < 3; ++k) {
      double fk = dw * v21[k];
      F[3 * i1 + k] = F[3 * i1 + k] - fk;
      F[3 * i2 + k] = F[3 * i2 + k] + fk;
    }
  }
}

// force_sumup.F90:66-333 (single thread: one buffer, so the thread
// reduction is the identity).
void force_sumup(orc_ctx &c, Rep &r, double *F) {
  std::fill(F, F + 3 * (size_t)c.nmp, 0.0);
  force_bond(c, r, F);
  force_fene(c, r, F);
  force_bangle(c, r, F);
  force_wca(c, r, F);
  if (c.nst > 0 || c.nhb > 0 || c.ntst > 0) {
    // force_sumup.F90:159-179: tertiary stacks first (they set st_status)
    r.st_status.assign(c.nst, 1);
    if (c.ntst > 0) dtrna_stack_nlocal(c, r, F);
    force_dtrna_stack(c, r, F);
    force_dtrna_hbond15(c, r, F);
  }
  force_exv_dt15(c, r, F);
  if (c.par.i_ele == TIS_ELE_DH) force_ele_DH(c, r, F);
  else if (c.par.i_ele == TIS_ELE_EWALD) force_ele_ewald(c, r, F);
  else if (c.par.i_ele == TIS_ELE_COULOMB) force_ele_coulomb(c, r, F);
}

// ------------------------------------------------------------- energies
// energy_bond.F90 / util_bondangle.F90 / energy_bangle.F90
double energy_bond(const orc_ctx &c, const Rep &r) {
  double e = 0;
  for (int ibd = 0; ibd < c.nbd; ++ibd) {
    int i1 = c.ibd2mp[2 * ibd] - 1, i2 = c.ibd2mp[2 * ibd + 1] - 1;
    double v[3];
    for (int k = 0; k < 3; ++k) v[k] = r.xyz[3 * i2 + k] - r.xyz[3 * i1 + k];
    double dist = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    double dd = dist - c.bd_nat[ibd];
    e += c.coef_bd[ibd] * (dd * dd);
  }
  return e;
}
double energy_bangle(const orc_ctx &c, const Rep &r) {
  double e = 0;
  for (int iba = 0; iba < c.nba; ++iba) {
    int i1 = c.iba2mp[3 * iba] - 1, i2 = c.iba2mp[3 * iba + 1] - 1, i3 = c.iba2mp[3 * iba + 2] - 1;
    double v21[3], v32[3];
    for (int k = 0; k < 3; ++k) {
      v21[k] = r.xyz[3 * i2 + k] - r.xyz[3 * i1 + k];
      v32[k] = r.xyz[3 * i3 + k] - r.xyz[3 * i2 + k];
    }
    double c11 = v21[0] * v21[0] + v21[1] * v21[1] + v21[2] * v21[2];
    double c22 = v32[0] * v32[0] + v32[1] * v32[1] + v32[2] * v32[2];
    double c21 = v32[0] * v21[0] + v32[1] * v21[1] + v32[2] * v21[2];
    double co = -c21 / std::sqrt(c11 * c22);
    if (co > 1.0) co = 1.0; else if (co < -1.0) co = -1.0;
    double dba = std::acos(co) - c.ba_nat[iba];
    e += c.coef_ba[iba] * (dba * dba);
  }
  return e;
}
double energy_fene(const orc_ctx &c, const Rep &r) {
  // energy_fene.F90: -k/2 * R0^2 * log(1 - (dr/R0)^2) with R0^2 = dist2_fene
  double e = 0;
  for (int i = 0; i < c.nfene; ++i) {
    int i1 = c.fene2mp[2 * i] - 1, i2 = c.fene2mp[2 * i + 1] - 1;
    double v[3];
    for (int k = 0; k < 3; ++k) v[k] = r.xyz[3 * i2 + k] - r.xyz[3 * i1 + k];
    double dd = norm2_3(v) - c.fene_nat[i];
    e += -0.5 * c.coef_fene[i] * c.dist2_fene[i] * std::log(1.0 - dd * dd / c.dist2_fene[i]);
  }
  return e;
}
// energy_wca.F90 (loop body): repulsive and attractive parts
void energy_wca(const orc_ctx &c, const Rep &r, double &e_rep, double &e_att) {
  double rcut_off2 = 1.0 / sq(c.par.wca_coef_cutoff);
  const bool peri = c.par.i_periodic == 1;
  e_rep = 0.0; e_att = 0.0;
  for (int i = 0; i < c.nwca; ++i) {
    int i1 = c.wca2mp[2 * i] - 1, i2 = c.wca2mp[2 * i + 1] - 1;
    double v21[3];
    if (!peri) for (int k = 0; k < 3; ++k) v21[k] = r.xyz[3 * i2 + k] - r.xyz[3 * i1 + k];
    else { for (int k = 0; k < 3; ++k) v21[k] = r.pxyz[3 * i2 + k] - r.pxyz[3 * i1 + k]; pbneighbor(c, v21, nullptr); }
    double dist2 = dot3(v21, v21);
    double ro2 = c.wca_nat[i] * c.wca_nat[i] / dist2;
    if (ro2 < rcut_off2) continue;
    double ro6 = std::pow(ro2, 6), ro3 = std::pow(ro2, 3);
    if (ro2 >= 1.0e0) {
      e_rep += c.coef_wca[i] * (ro6 - 2.0e0 * ro3 + 1.0e0);
      e_att += -c.coef_wca[c.nwca + i];
    } else {
      e_att += c.coef_wca[c.nwca + i] * (ro6 - 2.0e0 * ro3);
    }
  }
}
// energy_dtrna_stack.F90 (loop body)
double energy_stack(const orc_ctx &c, const Rep &r) {
  const Label &L = c.lab[r.label - 1];
  double e = 0;
  for (int ist = 0; ist < c.nst; ++ist) {
    if (!r.st_status.empty() && !r.st_status[ist]) continue;
    const int *m7 = &c.st2mp[7 * ist];
    auto X = [&](int k, int d) { return r.xyz[3 * (m7[k] - 1) + d]; };
    double v21[3], v34[3], v54[3], v56[3], v76[3];
    for (int d = 0; d < 3; ++d) {
      v21[d] = X(1, d) - X(0, d); v34[d] = X(2, d) - X(3, d); v54[d] = X(4, d) - X(3, d);
      v56[d] = X(4, d) - X(5, d); v76[d] = X(6, d) - X(5, d);
    }
    double ediv = 1.0;
    double dd = norm2_3(v21) - c.st_nat[3 * ist];
    ediv = ediv + c.st_coef[3 * ist] * dd * dd;
    double m[3], n[3];
    cross(v34, v54, m); cross(v54, v56, n);
    double dih = std::atan2(dot3(v34, n) * norm2_3(v54), dot3(m, n));
    double d = wrap_pi(dih - c.st_nat[3 * ist + 1]);
    ediv = ediv + c.st_coef[3 * ist + 1] * d * d;
    cross(v76, v56, m);
    for (int k = 0; k < 3; ++k) n[k] = -n[k];
    dih = std::atan2(dot3(v76, n) * norm2_3(v56), dot3(m, n));
    d = wrap_pi(dih - c.st_nat[3 * ist + 2]);
    ediv = ediv + c.st_coef[3 * ist + 2] * d * d;
    e += L.st_u0[ist] / ediv;
  }
  return e;
}
// energy_exv_dt15.F90:62-110
double energy_exv(const orc_ctx &c, const Rep &r) {
  double a = c.par.exv_adjust, e = 0;
  size_t nexv = r.iexv2mp.size() / 3;
  for (size_t k = 0; k < nexv; ++k) {
    int i1 = r.iexv2mp[3 * k] - 1, i2 = r.iexv2mp[3 * k + 1] - 1, im = r.iexv2mp[3 * k + 2] - 1;
    double dij = exv_dij(c, i1, i2);
    double v[3];
    for (int d = 0; d < 3; ++d) v[d] = r.pxyz[3 * i2 + d] - r.pxyz[3 * i1 + d] + c.d_mirror[im][d];
    double dist = norm2_3(v);
    if (dist > dij) continue;
    dist = dist + a - dij;
    double ene;
    if (dist > c.par.exv_inf) {
      double ro = a / dist;
      ene = c.exv_epsilon[i1] * c.exv_epsilon[i2] * (std::pow(ro, 12) - 2 * std::pow(ro, 6) + 1.0e0);
    } else ene = HIGH_ENERGY;
    e += ene;
  }
  return e;
}
// energy_ele_DH.F90:33-119 (i_temp_independent = 0)
double energy_DH(const orc_ctx &c, const Rep &r) {
  const Label &L = c.lab[r.label - 1];
  double cutoff2 = (c.par.i_DH_cutoff_type == 0) ? sq(c.par.cutoff_ele * L.cdist) : sq(c.par.cutoff_ele);
  double rcdist = 1.0 / L.cdist, e = 0;
  size_t nele = r.coef_ele.size();
  for (size_t k = 0; k < nele; ++k) {
    int i1 = r.iele2mp[4 * k] - 1, i2 = r.iele2mp[4 * k + 1] - 1, im = r.iele2mp[4 * k + 2] - 1;
    double v[3];
    for (int d = 0; d < 3; ++d) v[d] = r.pxyz[3 * i2 + d] - r.pxyz[3 * i1 + d] + c.d_mirror[im][d];
    double dist2 = dot3(v, v);
    if (dist2 > cutoff2) continue;
    double dist1 = std::sqrt(dist2);
    if (r.iele2mp[4 * k + 3] > 0 && !L.pmf_e.empty() && dist1 <= c.par.pmf_rmax) {
      // energy_ele_DH.F90:77-95: linear between the table points
      Rep &rw = const_cast<Rep &>(r);
      const int ib = pmf_bin(c, rw, dist1);
      e += L.pmf_e[ib] - L.pmf_f[ib] * (dist1 - (c.par.pmf_rmin + (double)ib * c.par.pmf_rbin));
      continue;
    }
    // coef_ele is rebuilt with the current label's coef (simu_para2.F90)
    int ic = c.lmp2charge[i1], jc = c.lmp2charge[i2];
    double ce = qch(c, L, ic) * qch(c, L, jc) * L.coef;
    e += ce / dist1 * std::exp(-dist1 * rcdist);
  }
  return e;
}
// energy_ele_coulomb.F90:31-70: coef_ele (1 / r - 1 / cutoff) inside the cutoff
double energy_coulomb(const orc_ctx &c, const Rep &r) {
  const Label &L = c.lab[r.label - 1];
  double cutoff2 = sq(c.par.cutoff_ele), cut_inv = 1.0e0 / c.par.cutoff_ele, e = 0;
  size_t nele = r.coef_ele.size();
  for (size_t k = 0; k < nele; ++k) {
    int i1 = r.iele2mp[4 * k] - 1, i2 = r.iele2mp[4 * k + 1] - 1, im = r.iele2mp[4 * k + 2] - 1;
    double v[3];
    for (int d = 0; d < 3; ++d) v[d] = r.pxyz[3 * i2 + d] - r.pxyz[3 * i1 + d] + c.d_mirror[im][d];
    double dist2 = dot3(v, v);
    if (dist2 > cutoff2) continue;
    double dist1 = std::sqrt(dist2);
    double ce = qch(c, L, c.lmp2charge[i1]) * qch(c, L, c.lmp2charge[i2]) * L.coef;
    e += ce * (1.0e0 / dist1 - cut_inv);
  }
  return e;
}
// energy_ele_coulomb_ewld.F90 (Fourier 75-89, real 137, self 212)
double energy_ewald(const orc_ctx &c, const Rep &r) {
  const Label &L = c.lab[r.label - 1];
  double e_f = 0.0;
  for (int ig = 0; ig < c.ewld_f_n; ++ig) {
    const double *k = &c.ewld_f_rlv[3 * ig];
    double scos = 0, ssin = 0;
    for (int ic = 0; ic < c.ncharge; ++ic) {
      int imp = c.icharge2mp[ic];
      double dp = dot3(k, &r.pxyz[3 * imp]);
      scos += qch(c, L, ic) * std::cos(dp);
      ssin += qch(c, L, ic) * std::sin(dp);
    }
    e_f += c.ewld_f_coef[ig] * (scos * scos + ssin * ssin);
  }
  double cutoff2 = sq(c.par.cutoff_ele), e_r = 0;
  size_t nele = r.coef_ele.size();
  for (size_t q = 0; q < nele; ++q) {
    int i1 = r.iele2mp[4 * q] - 1, i2 = r.iele2mp[4 * q + 1] - 1, im = r.iele2mp[4 * q + 2] - 1;
    double v[3];
    for (int d = 0; d < 3; ++d) v[d] = r.pxyz[3 * i2 + d] - r.pxyz[3 * i1 + d] + c.d_mirror[im][d];
    double dist2 = dot3(v, v);
    if (dist2 > cutoff2) continue;
    double dist1 = std::sqrt(dist2);
    double ce = qch(c, L, c.lmp2charge[i1]) * qch(c, L, c.lmp2charge[i2]) * L.coef;
    e_r += ce * std::erfc(c.par.ewld_alpha * dist1) / dist1;
  }
  double qq = 0;
  for (int ic = 0; ic < c.ncharge; ++ic) qq += qch(c, L, ic) * qch(c, L, ic);
  double e_s = c.ewld_s_coef * qq;
  return L.coef * (e_f + e_s) + e_r;
}
// energy_dtrna_hbond15.F90: with flg_hb_energy set the energies of the last
// force call are summed; otherwise terms and pruning are recomputed.
// Secondary bonds go to HBOND_DTRNA, tertiary ('T') ones to THBOND_DTRNA
// (energy_dtrna_hbond15.F90:135-143).
void energy_hbond(orc_ctx &c, Rep &r, bool reuse, double &e_sec, double &e_ter) {
  if (!reuse) {
    hbond15_terms(c, r);
    hbond15_prune(c, r, false);
  }
  e_sec = 0;
  e_ter = 0;
  for (int ihb1 : r.ineigh2hb)
    if (!r.hb_status.empty() && r.hb_status[ihb1 - 1]) {
      if (c.hb_tert[ihb1 - 1]) e_ter += r.ene_hb[ihb1 - 1];
      else e_sec += r.ene_hb[ihb1 - 1];
    }
}

void energy_sumup(orc_ctx &c, Rep &r, double *E, bool reuse_hb) {
  for (int i = 0; i < TIS_ETYPE_MAX; ++i) E[i] = 0.0;
  // energy_kinetic.F90: 0.5 m v^2
  double ek = 0;
  for (int imp = 0; imp < c.nmp; ++imp)
    ek += 0.5 * c.cmass[imp] * (sq(r.velo[3 * imp]) + sq(r.velo[3 * imp + 1]) + sq(r.velo[3 * imp + 2]));
  E[TIS_E_VELO - 1] = ek;
  E[TIS_E_BOND - 1] = energy_bond(c, r) + energy_fene(c, r);   // energy_fene.F90 adds to E_TYPE%BOND
  if (c.nwca) energy_wca(c, r, E[TIS_E_WCA_REP - 1], E[TIS_E_WCA_ATT - 1]);
  E[TIS_E_BANGLE - 1] = energy_bangle(c, r);
  if (c.nst > 0 || c.nhb > 0 || c.ntst > 0) {
    // energy_sumup.F90:197-215: the tertiary stacks set st_status first
    r.st_status.assign(c.nst, 1);
    if (c.ntst > 0) E[TIS_E_TSTACK_DTRNA - 1] = dtrna_stack_nlocal(c, r, nullptr);
    E[TIS_E_STACK_DTRNA - 1] = energy_stack(c, r);
    energy_hbond(c, r, reuse_hb, E[TIS_E_HBOND_DTRNA - 1], E[TIS_E_THBOND_DTRNA - 1]);
  }
  E[TIS_E_EXV_DT15 - 1] = energy_exv(c, r);
  if (c.par.i_ele == TIS_ELE_DH) E[TIS_E_ELE - 1] = energy_DH(c, r);
  else if (c.par.i_ele == TIS_ELE_EWALD) E[TIS_E_ELE - 1] = energy_ewald(c, r);
  else if (c.par.i_ele == TIS_ELE_COULOMB) E[TIS_E_ELE - 1] = energy_coulomb(c, r);
  double tot = 0;
  for (int i = 1; i <= TIS_ETYPE_MAX; ++i) {
    if (i == TIS_E_TOTAL || i == TIS_E_VELO) continue;
    tot += E[i - 1];
  }
  E[TIS_E_TOTAL - 1] = tot;
}

// mloop_ewld.F90:56-156
void setup_ewald(orc_ctx &c) {
  double alpha = c.par.ewld_alpha, hmax = c.par.ewld_hmax, L = c.par.psize[0];
  int lmax = (int)std::ceil(hmax);
  double hmax2 = hmax * hmax;
  std::vector<double> h, h2;
  for (int ix = -lmax; ix <= lmax; ++ix)
    for (int iy = -lmax; iy <= lmax; ++iy)
      for (int iz = -lmax; iz <= lmax; ++iz) {
        if (ix == 0 && iy == 0 && iz == 0) continue;
        double v[3] = {(double)ix, (double)iy, (double)iz};
        double r2 = dot3(v, v);
        if (r2 <= hmax2) { h.push_back(v[0]); h.push_back(v[1]); h.push_back(v[2]); h2.push_back(r2); }
      }
  int n = (int)h2.size();
  // comb sort by |h|^2 (mloop_ewld.F90:104-125)
  int icomb = n;
  bool swp = false;
  while (icomb > 1 || swp) {
    icomb = (icomb * 10) / 13;
    if (icomb < 1) icomb = 1;
    else if (icomb == 9 || icomb == 10) icomb = 11;
    swp = false;
    for (int i = 0; i < n - icomb; ++i) {
      if (h2[i] > h2[i + icomb]) {
        std::swap(h2[i], h2[i + icomb]);
        for (int d = 0; d < 3; ++d) std::swap(h[3 * i + d], h[3 * (i + icomb) + d]);
        swp = true;
      }
    }
  }
  double factor = 2.0 * F_PI / L;
  c.ewld_f_n = n;
  c.ewld_f_coef.resize(n);
  c.ewld_f_rlv.resize(3 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    c.ewld_f_coef[i] = 2.0 * F_PI / (L * L * L) * std::exp(-(factor * factor) * h2[i] / (4.0 * alpha * alpha)) /
                       ((factor * factor) * h2[i]);
    for (int d = 0; d < 3; ++d) c.ewld_f_rlv[3 * i + d] = factor * h[3 * i + d];
  }
  c.ewld_s_coef = -alpha / std::sqrt(F_PI);
}

bool take_noise_step(orc_ctx &c, std::vector<double> &rbm) {
  size_t per = 3 * (size_t)c.nmp * c.nrep;
  rbm.assign(per, 0.0);
  if (c.noise_pos < c.noise_nsteps) {
    std::memcpy(rbm.data(), &c.noise[per * c.noise_pos], per * sizeof(double));
    c.noise_pos++;
    return true;
  }
  c.noise_exhausted = true;
  return false;
}

double rlan1(const orc_ctx &c, int imp, double tempk) {
  // time_integral_pre.F90:166-167
  return std::sqrt(2.0e0 * c.fric[imp] * BOLTZ_KCAL_MOL * tempk / (c.par.tstep * c.cmass[imp]));
}

} // namespace

// ===================================================================== ABI
extern "C" {

orc_ctx *orc_create(const tis_topology *t, const tis_params *p, int nrep, const double *tempk) {
  orc_ctx *c = new orc_ctx();
  c->par = *p;
  c->nmp = t->nmp; c->nunit = t->nunit;
  c->lunit2mp.assign(t->lunit2mp, t->lunit2mp + 2 * t->nunit);
  c->iclass_unit.assign(t->iclass_unit, t->iclass_unit + t->nunit);
  c->imp2type.assign(t->imp2type, t->imp2type + t->nmp);
  c->imp2unit.assign(t->nmp, 0);
  c->iclass_mp.assign(t->nmp, 0);
  for (int u = 0; u < t->nunit; ++u)
    for (int i = t->lunit2mp[2 * u] - 1; i <= t->lunit2mp[2 * u + 1] - 1; ++i) {
      c->imp2unit[i] = u; c->iclass_mp[i] = t->iclass_unit[u];
    }
  c->cmass.assign(t->cmass, t->cmass + t->nmp);
  c->fric.assign(t->fric, t->fric + t->nmp);
  c->exv_radius.assign(t->exv_radius, t->exv_radius + t->nmp);
  c->exv_epsilon.assign(t->exv_epsilon, t->exv_epsilon + t->nmp);
  if (t->radius) c->radius.assign(t->radius, t->radius + t->nmp);
  else c->radius.assign(t->nmp, p->hi_radius);
  c->rcmass.resize(t->nmp);
  for (int i = 0; i < t->nmp; ++i) c->rcmass[i] = 1.0e0 / c->cmass[i];
  c->ncharge = t->ncharge;
  c->icharge2mp.resize(t->ncharge);
  c->lmp2charge.assign(t->nmp, -1);
  for (int i = 0; i < t->ncharge; ++i) { c->icharge2mp[i] = t->icharge2mp[i] - 1; c->lmp2charge[c->icharge2mp[i]] = i; }
  c->coef_charge.assign(t->coef_charge, t->coef_charge + t->ncharge);
  c->dt19 = p->i_dtrna_model == 2019;
  c->n_mg = 0;
  for (int i = 0; i < t->nmp; ++i) c->n_mg += (t->imp2type[i] == TIS_MP_ION_MG) ? 1 : 0;
  c->q_kind.assign(t->ncharge, 0);
  for (int i = 0; i < t->ncharge; ++i)   // simu_ele_set.F90:150-166
    c->q_kind[i] = (p->i_charge == 1 && t->imp2type[t->icharge2mp[i] - 1] == TIS_MP_RNA_PHOS &&
                    !(t->flg_charge_fixed && t->flg_charge_fixed[i])) ? 1 : 0;
  if (c->dt19 && c->n_mg > 0 && p->pmf_mg_p && p->pmf_nbin > 1) c->pmf.assign(p->pmf_mg_p, p->pmf_mg_p + p->pmf_nbin);
  c->par.pmf_mg_p = nullptr;   // borrowed by the caller; the copy above is the ctx's
  c->nbd = t->nbd; c->ibd2mp.assign(t->ibd2mp, t->ibd2mp + 2 * t->nbd);
  c->bd_nat.assign(t->bd_nat, t->bd_nat + t->nbd); c->coef_bd.assign(t->coef_bd, t->coef_bd + t->nbd);
  c->nba = t->nba; c->iba2mp.assign(t->iba2mp, t->iba2mp + 3 * t->nba);
  c->ba_nat.assign(t->ba_nat, t->ba_nat + t->nba); c->coef_ba.assign(t->coef_ba, t->coef_ba + t->nba);
  c->nst = t->nst;
  c->st2mp.assign(t->idtrna_st2mp, t->idtrna_st2mp + 7 * t->nst);
  c->st_nat.assign(t->dtrna_st_nat, t->dtrna_st_nat + 3 * t->nst);
  c->st_coef.assign(t->coef_dtrna_st, t->coef_dtrna_st + 3 * t->nst);
  c->st_hsTm.assign(t->dtrna_st_hsTm, t->dtrna_st_hsTm + 3 * t->nst);
  c->nhb = t->nhb;
  c->hb2mp.assign(t->idtrna_hb2mp, t->idtrna_hb2mp + 6 * t->nhb);
  c->hb_nat.assign(t->dtrna_hb_nat, t->dtrna_hb_nat + 6 * t->nhb);
  c->hb_coef.assign(t->coef_dtrna_hb, t->coef_dtrna_hb + 7 * t->nhb);
  c->hb_tert.assign(t->nhb, 0);
  for (int ihb = 0; ihb < t->nhb; ++ihb) c->hb_tert[ihb] = (t->flg_hb_tertiary && t->flg_hb_tertiary[ihb]) ? 1 : 0;
  c->hb2site.assign(t->idtrna_hb2hbsite, t->idtrna_hb2hbsite + 6 * t->nhb);
  c->nhbsite = t->nhbsite;
  c->nvalence.assign(t->nvalence_hbsite, t->nvalence_hbsite + t->nhbsite);
  c->hb_at_site.assign(t->nhbsite, {});
  for (int ihb = 0; ihb < t->nhb; ++ihb)
    for (int i = 0; i < 6; ++i) {   // neighbor_list_hb.F90:394-410 order: side1 slot i, side2 slot i
      int k = (i % 2 == 0) ? (i / 2) : (3 + i / 2);
      int s = c->hb2site[6 * ihb + k];
      if (s > 0) c->hb_at_site[s - 1].push_back(ihb + 1);
    }
  c->nfene = t->nfene;
  if (t->nfene) {
    c->fene2mp.assign(t->ifene2mp, t->ifene2mp + 2 * t->nfene);
    c->fene_nat.assign(t->fene_nat, t->fene_nat + t->nfene);
    c->coef_fene.assign(t->coef_fene, t->coef_fene + t->nfene);
    c->dist2_fene.assign(t->dist2_fene, t->dist2_fene + t->nfene);
  }
  c->ntst = t->ntst;
  if (t->ntst) {
    c->tst2mp.assign(t->idtrna_tst2mp, t->idtrna_tst2mp + 6 * t->ntst);
    c->tst_nat.assign(t->dtrna_tst_nat, t->dtrna_tst_nat + 6 * t->ntst);
    c->tst_coef.assign(t->coef_dtrna_tst, t->coef_dtrna_tst + 7 * t->ntst);
    c->tst2st.assign(2 * t->ntst, -1);
    c->tst_excl.assign(2 * t->ntst, 0);
    // mloop_dtrna.F90:74-140: side s of a tertiary stack is the secondary
    // stack between its base B and B - 3 (side 1) or B + 3 (side 2); without
    // such a stack the side is not exclusive
    for (int itst = 0; itst < t->ntst; ++itst)
      for (int sd = 0; sd < 2; ++sd) {
        const int imp1 = t->idtrna_tst2mp[6 * itst + sd];
        const int imp2 = (t->idtrna_tst2side[2 * itst + sd] == 1) ? imp1 - 3 : imp1 + 3;
        int found = -1;
        for (int ist = 0; ist < t->nst; ++ist) {
          const int a1 = t->idtrna_st2mp[7 * ist], a2 = t->idtrna_st2mp[7 * ist + 1];
          if ((imp1 == a1 && imp2 == a2) || (imp1 == a2 && imp2 == a1)) { found = ist; break; }
        }
        c->tst2st[2 * itst + sd] = found;
        c->tst_excl[2 * itst + sd] = (found >= 0 && t->flg_tst_exclusive[2 * itst + sd]) ? 1 : 0;
      }
  }
  c->nwca = t->nwca;
  if (t->nwca) {
    c->wca2mp.assign(t->iwca2mp, t->iwca2mp + 2 * t->nwca);
    c->wca_nat.assign(t->wca_nat, t->wca_nat + t->nwca);
    c->coef_wca.assign(t->coef_wca, t->coef_wca + 2 * t->nwca);
  }
  // mloop_neigh_dist.F90:28-149 (EXV_DT15 only)
  c->rneighbordist2_unit.assign(c->nunit * c->nunit, 0.0);
  for (int u = 0; u < c->nunit; ++u)
    for (int v = 0; v < c->nunit; ++v) {
      double max_cut = 0.0;
      if (c->iclass_unit[u] == TIS_CLASS_RNA && c->iclass_unit[v] == TIS_CLASS_RNA) {
        if (p->exv_dist > max_cut) max_cut = p->exv_dist;
        if (p->exv_dist_PS > max_cut) max_cut = p->exv_dist_PS;
      } else {
        for (int i = c->lunit2mp[2 * u] - 1; i <= c->lunit2mp[2 * u + 1] - 1; ++i)
          for (int j = c->lunit2mp[2 * v] - 1; j <= c->lunit2mp[2 * v + 1] - 1; ++j) {
            double cut = c->exv_radius[i] + c->exv_radius[j];
            if (cut > max_cut) max_cut = cut;
          }
      }
      c->rneighbordist2_unit[u * c->nunit + v] = sq(max_cut + p->neigh_margin);
    }
  // setp_periodic.F90:78-113 (zero table when not periodic: setpara.F90:42)
  for (int i = 0; i < 3; ++i) c->psizeh[i] = p->psize[i] / 2.0;
  int im = 0;
  for (int ix = 1; ix <= 3; ++ix)
    for (int iy = 1; iy <= 3; ++iy)
      for (int iz = 1; iz <= 3; ++iz) {
        int idx[3] = {ix, iy, iz};
        for (int d = 0; d < 3; ++d) {
          double v = 0.0;
          if (p->i_periodic == 1) v = (idx[d] == 1) ? -p->psize[d] : (idx[d] == 2 ? p->psize[d] : 0.0e0);
          c->d_mirror[im][d] = v;
        }
        ++im;
      }
  // mloop_dtrna.F90:149-152 (i_neigh_dynamic = 1)
  c->hb_neigh_dist2.resize(c->nhb);
  for (int ihb = 0; ihb < c->nhb; ++ihb)
    c->hb_neigh_dist2[ihb] = sq(c->hb_nat[6 * ihb] + p->hb_cutoff_dist + p->neigh_margin);
  // simu_para.F90:26-27
  c->tstep2 = 0.5e0 * p->tstep * p->tstep;
  c->tsteph = 0.5e0 * p->tstep;
  if (p->i_ele == TIS_ELE_EWALD) setup_ewald(*c);
  // replicas and labels
  c->nrep = nrep;
  c->rep.resize(nrep);
  c->lab.resize(nrep);
  c->lab2rep.resize(nrep);
  for (int l = 0; l < nrep; ++l) {
    c->lab[l].tempk = tempk[l];
    ele_set(*c, c->lab[l]);
    set_dtrna(*c, c->lab[l]);
    c->lab2rep[l] = l + 1;
  }
  for (int i = 0; i < nrep; ++i) {
    Rep &r = c->rep[i];
    r.label = i + 1;
    size_t n3 = 3 * (size_t)c->nmp;
    r.xyz.assign(n3, 0); r.pxyz.assign(n3, 0); r.velo.assign(n3, 0);
    r.accel.assign(n3, 0); r.force.assign(n3, 0); r.dxyz.assign(n3, 0);
    r.st_status.assign(c->nst, 1);
  }
  para2(*c);
  return c;
}

void orc_destroy(orc_ctx *c) { delete c; }

int orc_set_state(orc_ctx *c, const double *xyz, const double *velo, const double *accel) {
  size_t n3 = 3 * (size_t)c->nmp;
  for (int i = 0; i < c->nrep; ++i) {
    Rep &r = c->rep[i];
    std::memcpy(r.xyz.data(), xyz + n3 * i, n3 * sizeof(double));
    r.pxyz = r.xyz;
    if (velo) std::memcpy(r.velo.data(), velo + n3 * i, n3 * sizeof(double));
    else std::fill(r.velo.begin(), r.velo.end(), 0.0);
    if (accel) std::memcpy(r.accel.data(), accel + n3 * i, n3 * sizeof(double));
    else std::fill(r.accel.begin(), r.accel.end(), 0.0);
    std::fill(r.dxyz.begin(), r.dxyz.end(), 0.0);
  }
  return 0;
}

int orc_get_state(orc_ctx *c, double *xyz, double *velo, double *accel) {
  size_t n3 = 3 * (size_t)c->nmp;
  for (int i = 0; i < c->nrep; ++i) {
    if (xyz) std::memcpy(xyz + n3 * i, c->rep[i].xyz.data(), n3 * sizeof(double));
    if (velo) std::memcpy(velo + n3 * i, c->rep[i].velo.data(), n3 * sizeof(double));
    if (accel) std::memcpy(accel + n3 * i, c->rep[i].accel.data(), n3 * sizeof(double));
  }
  return 0;
}

int orc_get_pxyz(orc_ctx *c, double *pxyz) {
  size_t n3 = 3 * (size_t)c->nmp;
  for (int i = 0; i < c->nrep; ++i) std::memcpy(pxyz + n3 * i, c->rep[i].pxyz.data(), n3 * sizeof(double));
  return 0;
}

int orc_set_noise(orc_ctx *c, const double *noise, int nsteps, const double *unif, int nunif) {
  size_t per = 3 * (size_t)c->nmp * c->nrep;
  c->noise.assign(noise, noise + per * (size_t)nsteps);
  c->noise_nsteps = nsteps;
  c->noise_pos = 0;
  c->noise_exhausted = false;
  for (int i = 0; i < c->nrep; ++i) {
    Rep &r = c->rep[i];
    if (unif) r.unif.assign(unif + (size_t)nunif * i, unif + (size_t)nunif * (i + 1));
    else r.unif.clear();
    r.upos = 0;
    r.unif_exhausted = false;
  }
  return 0;
}

int orc_neighbor(orc_ctx *c, int irep) {
  if (irep < 0) { for (auto &r : c->rep) neighbor(*c, r); }
  else neighbor(*c, c->rep[irep - 1]);
  return 0;
}

int orc_get_exv_list(orc_ctx *c, int irep, int *out, int cap) {
  const Rep &r = c->rep[irep - 1];
  int n = (int)(r.iexv2mp.size() / 3);
  if (out) std::memcpy(out, r.iexv2mp.data(), sizeof(int) * 3 * (size_t)std::min(n, cap));
  return n;
}
int orc_get_ele_list(orc_ctx *c, int irep, int *out, double *coef, int cap) {
  const Rep &r = c->rep[irep - 1];
  int n = (int)r.coef_ele.size();
  int m = std::min(n, cap);
  if (out) std::memcpy(out, r.iele2mp.data(), sizeof(int) * 4 * (size_t)m);
  if (coef) std::memcpy(coef, r.coef_ele.data(), sizeof(double) * (size_t)m);
  return n;
}
int orc_get_hb_list(orc_ctx *c, int irep, int *out, int cap) {
  const Rep &r = c->rep[irep - 1];
  int n = (int)r.ineigh2hb.size();
  if (out) std::memcpy(out, r.ineigh2hb.data(), sizeof(int) * (size_t)std::min(n, cap));
  return n;
}
int orc_get_hb_status(orc_ctx *c, int irep, int *status, double *ene) {
  const Rep &r = c->rep[irep - 1];
  for (int i = 0; i < c->nhb; ++i) {
    if (status) status[i] = r.hb_status.empty() ? 0 : r.hb_status[i];
    if (ene) ene[i] = r.ene_hb.empty() ? 0.0 : r.ene_hb[i];
  }
  return c->nhb;
}

int orc_force_sumup(orc_ctx *c, int irep, double *force) {
  Rep &r = c->rep[irep - 1];
  force_sumup(*c, r, r.force.data());
  if (force) std::memcpy(force, r.force.data(), 3 * (size_t)c->nmp * sizeof(double));
  return r.unif_exhausted ? TIS_E_NOISE_EXHAUSTED : 0;
}

// Single force term for tests: term = 0 bond, 1 angle, 2 stack, 3 hbond, 4 exv, 5 DH, 6 Ewald, 7 fene, 8 wca, 9 tertiary stack, 10 Coulomb.
int orc_force_term(orc_ctx *c, int irep, int term, double *force) {
  Rep &r = c->rep[irep - 1];
  std::fill(force, force + 3 * (size_t)c->nmp, 0.0);
  switch (term) {
    case 0: force_bond(*c, r, force); break;
    case 1: force_bangle(*c, r, force); break;
    case 2:   // st_status as force_sumup sets it
      if (c->ntst > 0) dtrna_stack_nlocal(*c, r, nullptr);
      else r.st_status.assign(c->nst, 1);
      force_dtrna_stack(*c, r, force);
      break;
    case 3: force_dtrna_hbond15(*c, r, force); break;
    case 4: force_exv_dt15(*c, r, force); break;
    case 5: force_ele_DH(*c, r, force); break;
    case 6: force_ele_ewald(*c, r, force); break;
    case 10: force_ele_coulomb(*c, r, force); break;
    case 7: force_fene(*c, r, force); break;
    case 8: force_wca(*c, r, force); break;
    case 9: dtrna_stack_nlocal(*c, r, force); break;
    default: return TIS_E_ARG;
  }
  return 0;
}

int orc_energy_sumup(orc_ctx *c, int irep, double *energy, int reuse_hb) {
  energy_sumup(*c, c->rep[irep - 1], energy, reuse_hb != 0);
  return 0;
}

// simu_hydro_tensors.F90:139-182 (HI_TENSOR%RPY, one radius) and 304-324
// (Cholesky); D and L are (3N, 3N) column-major.  Returns 0 or TIS_E_NOT_SPD.
int hydro_tensors(const orc_ctx *c, const Rep &r, double *D, double *Lc) {
  double tempk = c->lab[r.label - 1].tempk;
  int N = c->nmp, n = 3 * N;
  double c6 = BOLTZ_KCAL_MOL * tempk / (6.0e0 * F_PI * c->par.viscosity);
  double c8 = BOLTZ_KCAL_MOL * tempk / (8.0e0 * F_PI * c->par.viscosity);
  const int type = c->par.i_hydro_tensor == 0 ? TIS_HI_RPY : c->par.i_hydro_tensor;
  const double rad = c->radius[0];   // radius(1): RPY, RPY_OVER, ERMAK_OVER
  auto Dm = [&](int i, int j) -> double & { return D[(size_t)j * n + i]; };
  std::fill(D, D + (size_t)n * n, 0.0);
  for (int i = 0; i < N; ++i) {
    int i0 = 3 * i;
    const double rad_i = c->radius[i];
    for (int j = i + 1; j < N; ++j) {
      int j0 = 3 * j;
      const double rad_j = c->radius[j];
      double rv[3];
      for (int d = 0; d < 3; ++d) rv[d] = r.xyz[3 * j + d] - r.xyz[3 * i + d];
      double r_sq = dot3(rv, rv), r_abs = std::sqrt(r_sq);
      double pre1, pre2;
      bool diag_only = false;
      if (type == TIS_HI_ZUK_RPY) {   // simu_hydro_tensors.F90:50-124
        if ((rad_i + rad_j) < r_abs) {
          double rad_i_sq = rad_i * rad_i, rad_j_sq = rad_j * rad_j;
          pre1 = c8 / r_abs * (1.0 + (rad_i_sq + rad_j_sq) / (3.0 * r_sq));
          pre2 = c8 / r_abs * (1.0 - (rad_i_sq + rad_j_sq) / r_sq) / r_sq;
        } else {
          double rad_s, rad_l;
          if (rad_i < rad_j) { rad_s = rad_i; rad_l = rad_j; } else { rad_s = rad_j; rad_l = rad_i; }
          if ((rad_l - rad_s) < r_abs) {
            double r_cb = r_sq * r_abs;
            double dr2 = (rad_i - rad_j) * (rad_i - rad_j);
            double y1 = dr2 + 3 * r_sq, y2 = dr2 - r_sq;
            pre1 = c6 / rad_i / rad_j * (16.0 * r_cb * (rad_i + rad_j) - y1 * y1) / 32.0 / r_cb;
            pre2 = c6 / rad_i / rad_j * 3.0 * (y2 * y2) / 32.0 / r_cb / r_sq;
          } else {
            pre1 = c6 / rad_l; pre2 = 0.0;
            diag_only = true;
          }
        }
      } else if (type == TIS_HI_RPY || 2.0 * rad < r_abs) {   // :139-182, and the far pairs of :187-300
        double rad_sq = rad * rad;
        pre1 = c8 / r_abs * (1.0 + 2.0 * rad_sq / (3.0 * r_sq));
        pre2 = c8 / r_abs * (1.0 - 2.0 * rad_sq / r_sq) / r_sq;
      } else if (type == TIS_HI_RPY_OVER) {   // :216-217
        pre1 = c6 / rad * (1.0 - 9.0 / 32.0 * r_abs / rad);
        pre2 = c6 / rad * 3.0 / 32.0 / rad / r_abs;
      } else {   // ERMAK_OVER :269-270
        pre1 = c8 / 2.0 / rad * 7.0 / 6.0;
        pre2 = c8 / 2.0 / 2.0 / r_sq;
      }
      for (int ii = 0; ii < 3; ++ii) {
        if (diag_only) { Dm(i0 + ii, j0 + ii) = pre1; continue; }
        Dm(i0 + ii, j0 + ii) = pre1 + pre2 * rv[ii] * rv[ii];
        for (int jj = ii + 1; jj < 3; ++jj) {
          Dm(i0 + ii, j0 + jj) = pre2 * rv[ii] * rv[jj];
          Dm(i0 + jj, j0 + ii) = Dm(i0 + ii, j0 + jj);
        }
      }
    }
  }
  // D = D + transpose(D)
  for (int j = 0; j < n; ++j)
    for (int i = j + 1; i < n; ++i) {
      double s = Dm(i, j) + Dm(j, i);
      Dm(i, j) = s; Dm(j, i) = s;
    }
  for (int i = 0; i < n; ++i) Dm(i, i) = c6 / (type == TIS_HI_ZUK_RPY ? c->radius[i / 3] : rad);
  if (!Lc) return 0;
  auto Lm = [&](int i, int j) -> double & { return Lc[(size_t)j * n + i]; };
  std::fill(Lc, Lc + (size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) {
    double x = Dm(i, i);
    for (int k = 0; k < i; ++k) x -= Lm(i, k) * Lm(i, k);
    if (x <= 0.0) return TIS_E_NOT_SPD;
    x = std::sqrt(x);
    Lm(i, i) = x;
    for (int j = i + 1; j < n; ++j) {
      double s = 0.0;
      for (int k = 0; k < i; ++k) s += Lm(j, k) * Lm(i, k);
      Lm(j, i) = (Dm(i, j) - s) / x;
    }
  }
  return 0;
}
// time_integral_pre.F90:75-180 (Langevin) and :313-317 (Brownian-HI:
// velocities zero, rlan_const(1) = tstep / kT, rlan_const(2) = sqrt(2 tstep))
int orc_time_integral_pre(orc_ctx *c) {
  for (auto &r : c->rep) neighbor(*c, r);
  for (auto &r : c->rep) std::fill(r.dxyz.begin(), r.dxyz.end(), 0.0);
  std::vector<double> rbm;
  take_noise_step(*c, rbm);
  if (c->par.i_simulate_type == TIS_SIM_BROWNIAN_HI) {
    for (auto &r : c->rep) {
      force_sumup(*c, r, r.force.data());
      std::fill(r.velo.begin(), r.velo.end(), 0.0);
      std::fill(r.accel.begin(), r.accel.end(), 0.0);
    }
    return c->noise_exhausted ? TIS_E_NOISE_EXHAUSTED : 0;
  }
  size_t n3 = 3 * (size_t)c->nmp;
  for (int i = 0; i < c->nrep; ++i) {
    Rep &r = c->rep[i];
    force_sumup(*c, r, r.force.data());
    double T = c->lab[r.label - 1].tempk;
    for (int imp = 0; imp < c->nmp; ++imp) {
      double c1 = rlan1(*c, imp, T);
      for (int d = 0; d < 3; ++d) {
        double rf = c1 * rbm[n3 * i + 3 * imp + d];
        r.accel[3 * imp + d] = r.force[3 * imp + d] * c->rcmass[imp] + rf;
      }
    }
  }
  return c->noise_exhausted ? TIS_E_NOISE_EXHAUSTED : 0;
}

// time_integral.F90:57-190 (Langevin), nsteps times
int orc_step(orc_ctx *c, long nsteps) {
  size_t n3 = 3 * (size_t)c->nmp;
  std::vector<double> rbm;
  for (long s = 0; s < nsteps; ++s) {
    for (auto &r : c->rep) {
      long istep = r.istep + 1;
      bool rebuild;
      if (c->par.n_step_neighbor <= 0) {
        double d2max = 0, d2max2 = 0;
        for (int imp = 0; imp < c->nmp; ++imp) {
          double d2 = dot3(&r.dxyz[3 * imp], &r.dxyz[3 * imp]);
          if (d2 > d2max) { d2max2 = d2max; d2max = d2; }
          else if (d2 > d2max2) d2max2 = d2;
        }
        rebuild = std::sqrt(d2max) + std::sqrt(d2max2) > c->par.neigh_margin;
      } else {
        rebuild = (istep % c->par.n_step_neighbor) == 1 || istep == 1;
      }
      if (rebuild) {
        neighbor(*c, r);
        r.last_rebuild = istep;   // the step whose trigger fired (outfile%neigh record, time_integral.F90:76-84)
        if (c->par.n_step_neighbor <= 0) std::fill(r.dxyz.begin(), r.dxyz.end(), 0.0);
      }
    }
    take_noise_step(*c, rbm);
    if (c->par.i_simulate_type == TIS_SIM_BROWNIAN_HI) {
      // time_integral.F90:429-457: D and L at the current x (every
      // n_step_hydro steps), dx = rlan1 D F + rlan2 L xi, then the force
      const int n = 3 * c->nmp;
      const int every = c->par.n_step_hydro > 0 ? c->par.n_step_hydro : 1;
      for (int i = 0; i < c->nrep; ++i) {
        Rep &r = c->rep[i];
        r.istep++;
        const double T = c->lab[r.label - 1].tempk;
        if ((r.istep - 1) % every == 0) {
          r.hD.resize((size_t)n * n);
          r.hL.resize((size_t)n * n);
          if (hydro_tensors(c, r, r.hD.data(), r.hL.data()) != 0) r.not_spd = 1;
        }
        const double rl1 = c->par.tstep / (BOLTZ_KCAL_MOL * T), rl2 = std::sqrt(2.0e0 * c->par.tstep);
        const double *xi = &rbm[n3 * i];
        for (int k = 0; k < n; ++k) {
          double df = 0.0, dr = 0.0;
          for (int m = 0; m < n; ++m) df += r.hD[(size_t)k * n + m] * r.force[m];
          for (int m = 0; m <= k; ++m) dr += r.hL[(size_t)m * n + k] * xi[m];
          const double dx = rl1 * df + rl2 * dr;
          r.xyz[k] = r.xyz[k] + dx;
          r.pxyz[k] = r.pxyz[k] + dx;
          r.dxyz[k] = r.dxyz[k] + dx;
        }
        force_sumup(*c, r, r.force.data());
      }
      continue;
    }
    for (int i = 0; i < c->nrep; ++i) {
      Rep &r = c->rep[i];
      r.istep++;
      double T = c->lab[r.label - 1].tempk;
      for (int imp = 0; imp < c->nmp; ++imp) {
        double tfh = 0.5e0 * c->par.tstep * c->fric[imp];
        double u1 = 1.0e0 - tfh;
        double c4 = c->par.tstep * u1;
        for (int d = 0; d < 3; ++d) {
          double dx = c4 * r.velo[3 * imp + d] + c->tstep2 * r.accel[3 * imp + d];
          r.xyz[3 * imp + d] = r.xyz[3 * imp + d] + dx;
          r.pxyz[3 * imp + d] = r.pxyz[3 * imp + d] + dx;
          r.dxyz[3 * imp + d] = r.dxyz[3 * imp + d] + dx;
        }
      }
      force_sumup(*c, r, r.force.data());
      for (int imp = 0; imp < c->nmp; ++imp) {
        double tfh = 0.5e0 * c->par.tstep * c->fric[imp];
        double u1 = 1.0e0 - tfh;
        double u2 = 1.0e0 - tfh + tfh * tfh;
        double c1 = rlan1(*c, imp, T), c2 = u1 * u2, c3 = c->tsteph * u1;
        for (int d = 0; d < 3; ++d) {
          double rf = c1 * rbm[n3 * i + 3 * imp + d];
          double af = r.force[3 * imp + d] * c->rcmass[imp] + rf;
          r.velo[3 * imp + d] = c2 * r.velo[3 * imp + d] + c3 * (r.accel[3 * imp + d] + af);
          r.accel[3 * imp + d] = af;
        }
      }
    }
  }
  return c->noise_exhausted ? TIS_E_NOISE_EXHAUSTED : 0;
}

// energy_allrep.F90:123-260 + simu_replica_exchange.F90:87-300 + the
// rlan_const / simu_para2 refresh (time_integral_post.F90:293-349).
// u[k] is random0(k); energies are recomputed (flg_hb_energy = .false.).
int orc_replica_exchange(orc_ctx *c, const double *u, int *n_accept) {
  int n = c->nrep;
  auto pair_of = [&](int l) -> int {   // exchange_pair_tb for one dimension
    if (c->idx_pair == 1) { if (l % 2 == 1) return (l + 1 <= n) ? l + 1 : 0; return l - 1; }
    if (l == 1) return 0;
    if (l % 2 == 0) return (l + 1 <= n) ? l + 1 : 0;
    return l - 1;
  };
  std::vector<double> e_own(n), e_opp(n);
  double E[TIS_ETYPE_MAX];
  for (int i = 0; i < n; ++i) {
    Rep &r = c->rep[i];
    // energy_allrep.F90:123-125 runs before flg_hb_energy is cleared: the
    // hbond energies of the last force call are reused
    energy_sumup(*c, r, E, true);
    e_own[i] = E[TIS_E_TOTAL - 1];
    int lo = pair_of(r.label);
    if (lo == 0 || lo > n) { e_opp[i] = 0.0; continue; }
    int keep = r.label;
    // evaluate at the partner label's temperature, then restore
    r.label = lo;
    c->beta_hbond15 = 1.0e0 / (c->lab[lo - 1].tempk * BOLTZ_KCAL_MOL);
    energy_sumup(*c, r, E, false);
    e_opp[i] = E[TIS_E_TOTAL - 1];
    r.label = keep;
    c->beta_hbond15 = 1.0e0 / (c->lab[keep - 1].tempk * BOLTZ_KCAL_MOL);
  }
  int nrand = 0, nacc = 0;
  for (int li = 1; li <= n; ++li) {
    int lj = pair_of(li);
    if (lj < li) continue;
    nrand++;
    int ri = c->lab2rep[li - 1], rj = c->lab2rep[lj - 1];
    double tm = c->lab[li - 1].tempk, tn = c->lab[lj - 1].tempk;
    double pim = e_own[ri - 1], pin = e_opp[ri - 1], pjn = e_own[rj - 1], pjm = e_opp[rj - 1];
    double delta = ((pjm - pim) / tm - (pjn - pin) / tn) / BOLTZ_KCAL_MOL;
    bool acc = delta < 0.0e0 || u[nrand - 1] <= std::exp(-delta);
    if (acc) {
      c->rep[ri - 1].label = lj; c->rep[rj - 1].label = li;
      c->lab2rep[li - 1] = rj; c->lab2rep[lj - 1] = ri;
      double sf = std::sqrt(tn / tm);
      for (auto &v : c->rep[ri - 1].velo) v = sf * v;
      for (auto &v : c->rep[rj - 1].velo) v = v / sf;
      nacc++;
    }
  }
  c->idx_pair = (c->idx_pair == 2) ? 1 : c->idx_pair + 1;
  para2(*c);
  if (n_accept) *n_accept = nacc;
  return 0;
}

// energy_allrep.F90:130-217 for replica irep alone: out2 = (energy at its
// own label with the hbond energies of the last force call, energy at the
// exchange partner's label or 0 without one), labels unchanged
int orc_replica_energy(orc_ctx *c, int irep, double *out2) {
  const int n = c->nrep;
  Rep &r = c->rep[irep - 1];
  double E[TIS_ETYPE_MAX];
  energy_sumup(*c, r, E, true);
  out2[0] = E[TIS_E_TOTAL - 1];
  int lo;
  if (c->idx_pair == 1) lo = (r.label % 2 == 1) ? ((r.label + 1 <= n) ? r.label + 1 : 0) : r.label - 1;
  else if (r.label == 1) lo = 0;
  else lo = (r.label % 2 == 0) ? ((r.label + 1 <= n) ? r.label + 1 : 0) : r.label - 1;
  if (lo == 0) { out2[1] = 0.0; return 0; }
  const int keep = r.label;
  const double bkeep = c->beta_hbond15;
  r.label = lo;
  c->beta_hbond15 = 1.0e0 / (c->lab[lo - 1].tempk * BOLTZ_KCAL_MOL);
  energy_sumup(*c, r, E, false);
  out2[1] = E[TIS_E_TOTAL - 1];
  r.label = keep;
  c->beta_hbond15 = bkeep;
  return 0;
}

// The outcome of an exchange decided elsewhere: the new rep2lab (1-based),
// velocities times vscale[r] (> 0) or divided by -vscale[r] (< 0), the pair
// alternation and the label-dependent parameters, as orc_replica_exchange
// leaves them.
int orc_rex_apply(orc_ctx *c, const int *rep2lab, const double *vscale) {
  for (int i = 0; i < c->nrep; ++i) {
    Rep &r = c->rep[i];
    r.label = rep2lab[i];
    c->lab2rep[rep2lab[i] - 1] = i + 1;
    if (vscale[i] > 0.0) for (auto &v : r.velo) v = vscale[i] * v;
    else if (vscale[i] < 0.0) for (auto &v : r.velo) v = v / (-vscale[i]);
  }
  c->idx_pair = (c->idx_pair == 2) ? 1 : c->idx_pair + 1;
  para2(*c);
  return 0;
}

int orc_get_labels(orc_ctx *c, int *rep2lab) {
  for (int i = 0; i < c->nrep; ++i) rep2lab[i] = c->rep[i].label;
  return 0;
}

// Per-label derived parameters for tests: ek, coef, cdist, beta_hbond15.
int orc_label_params(orc_ctx *c, int label, double *out4) {
  const Label &L = c->lab[label - 1];
  out4[0] = L.ek; out4[1] = L.coef; out4[2] = L.cdist; out4[3] = c->beta_hbond15;
  return 0;
}

int orc_ewald_table(orc_ctx *c, double *rlv, double *coef, int cap) {
  int n = c->ewld_f_n;
  int m = std::min(n, cap);
  if (rlv) std::memcpy(rlv, c->ewld_f_rlv.data(), sizeof(double) * 3 * (size_t)m);
  if (coef) std::memcpy(coef, c->ewld_f_coef.data(), sizeof(double) * (size_t)m);
  return n;
}

// Direct lattice sum of the Coulomb energy over (2*nlat+1)^3 images with
// the neutral-box convention of utility/coulomb_energy_exact.F90: every
// pair within the central box once, plus every image pair (i, j+nL, n != 0)
// with weight 1/2.  Returns coef(T) * sum q_i q_j / r.
double orc_coulomb_direct(orc_ctx *c, int irep, int nlat) {
  const Rep &r = c->rep[irep - 1];
  const Label &L = c->lab[r.label - 1];
  double e = 0.0;
  double Lb[3] = {c->par.psize[0], c->par.psize[1], c->par.psize[2]};
  for (int ia = -nlat; ia <= nlat; ++ia)
    for (int ib = -nlat; ib <= nlat; ++ib)
      for (int ic = -nlat; ic <= nlat; ++ic) {
        bool central = (ia == 0 && ib == 0 && ic == 0);
        // spherical summation order
        if (ia * ia + ib * ib + ic * ic > nlat * nlat) continue;
        double sh[3] = {ia * Lb[0], ib * Lb[1], ic * Lb[2]};
        for (int i = 0; i < c->ncharge; ++i) {
          int mi = c->icharge2mp[i];
          for (int j = 0; j < c->ncharge; ++j) {
            if (central && j <= i) continue;
            int mj = c->icharge2mp[j];
            double v[3];
            for (int d = 0; d < 3; ++d) v[d] = r.pxyz[3 * mj + d] + sh[d] - r.pxyz[3 * mi + d];
            double rr = norm2_3(v);
            double w = central ? 1.0 : 0.5;
            e += w * c->coef_charge[i] * c->coef_charge[j] / rr;
          }
        }
      }
  return L.coef * e;
}

int orc_hydro_tensors(orc_ctx *c, int irep, double *D, double *Lc) {
  return hydro_tensors(c, c->rep[irep - 1], D, Lc);
}

int orc_not_spd(orc_ctx *c) {
  int f = 0;
  for (auto &r : c->rep) f |= r.not_spd;
  return f;
}

// neighbour rebuilds of replica irep and the step of the last one
void orc_rebuild_info(orc_ctx *c, int irep, long *n, long *last) {
  const Rep &r = c->rep[irep - 1];
  if (n) *n = r.nrebuild;
  if (last) *last = r.last_rebuild;
}

long orc_nclamp(orc_ctx *c) {
  long s = 0;
  for (auto &r : c->rep) s += r.nclamp;
  return s;
}

int orc_pmf_range(orc_ctx *c) {
  int f = 0;
  for (auto &r : c->rep) f |= r.pmf_range;
  return f;
}

// Zp of a label and its Mg-P table (energy, force; n entries each).  Returns
// the table length, 0 when the label has none.
int orc_label_pmf(orc_ctx *c, int label, double *zp, double *e, double *f, int cap) {
  const Label &L = c->lab[label - 1];
  if (zp) *zp = L.zp;
  const int n = (int)L.pmf_e.size();
  for (int i = 0; i < std::min(n, cap); ++i) {
    if (e) e[i] = L.pmf_e[i];
    if (f) f[i] = L.pmf_f[i];
  }
  return n;
}

double orc_boltz_kcal_mol(void) { return BOLTZ_KCAL_MOL; }

} // extern "C"
