// pip_capi.cu -- C ABI of the two-fluid step (include/pip_gpu.h): context, host<->device
// copies and the device-side time loop.
//
// The context owns two device arrays of NV = nvm + 5 planes (A: current state / U0 / U2,
// B: U1), a small control block (DevCtrl) and lazily allocated scratch for the unit-level
// entry points.  pip_run keeps dt, time and the stop flags on the device and replays a
// captured CUDA graph of K steps (2 kernels per step) between host polls.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/pip_bench.h"
#include "../../include/pip_gpu.h"
#include "pip_kernels.cuh"

using pip::DevCtrl;
using pip::KParams;

static int g_last_cuda_error = 0;

struct pip_ctx {
  pip_params p{};
  std::vector<double> dx, dy, dz;
  KParams kp{};
  const pip::Launchers *L = nullptr;
  int device = 0;
  cudaStream_t stream = nullptr;
  double *A = nullptr, *B = nullptr;  // NV planes each (FP64 form; A stages the mixed form)
  float *Ahi = nullptr, *Alo = nullptr, *Bf = nullptr;  // FP32-mixed form
  CUtensorMap tm_a, tm_b;             // TMA maps of the stage sources (A and B, or Ahi and Bf)
  bool tma = false;                   // the maps exist (2D grids that meet the TMA rules)
  bool mixed = false;
  double *d_dx = nullptr, *d_dy = nullptr, *d_rdx = nullptr, *d_rdy = nullptr;
  double *scratch = nullptr;          // NV planes for pip_flux / pip_source
  int *d_flag = nullptr;
  DevCtrl *ctrl = nullptr;
  DevCtrl *h_ctrl = nullptr;          // pinned mirror
  pip::HcEngine *hc = nullptr;        // implicit conduction (flag_heat = 1)
  double *d_dt = nullptr;             // host dt of pip_step / pip_conduction on the device
  int hc_iters = 0;                   // BiCGstab iterations of the last run
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  int neighbor[4] = {-1, -1, -1, -1};  // set_mpi_neighbor: rank across each face, -1 physical
  bool exchanged = false;             // some face is filled by the halo exchange
  int last_stage = 0;                 // RK stage that wrote the state last (1: the U1 array)
  cudaStream_t halo_stream = nullptr; // pip_set_halo_stream: the stream of pack and unpack
  cudaStream_t rows_stream = nullptr; // pip_dev_stage_split: high-priority stream of the
  cudaEvent_t rows_ev[2] = {nullptr, nullptr};  // boundary rows, and its two events
  bool dev_loop = false;              // pip_dev_begin has set up the device-driven loop
  bool uploaded = false;
  double *acf = nullptr;              // alpha_c per cell (flag_col 2..7)
  double *etaf = nullptr;             // eta per cell (flag_resi 1)
  unsigned long long *d_resi = nullptr;  // cfl_resi's bound of the current eta (flag_resi 2)
  bool coef_valid = false;            // set_coefficients(U_h,U_m,0) has run on this state
  double *irg = nullptr;              // set_IR type 1's or type 4's rates (2 planes)
  // set_IR type 4: Nexcite (two sets of 6 planes, nl_cur the current), colrat (36 planes),
  // ion_pot, the table, the coefficients, the reference rates (37 values)
  double *nl_nex[2] = {nullptr, nullptr};
  int nl_cur = 0;
  double *nl_cr = nullptr, *nl_ip = nullptr, *nl_tab = nullptr, *nl_ref = nullptr;
  double *nl_rtab = nullptr;
  pip::NlevConst *nl_k = nullptr;
  bool nl_ready = false;              // pip_set_nlevel has run
  bool nl_init = false;               // the fresh-start block (Gm_rec_ref, ion_pot) has run
  double dt = 0.0, cmax = 0.0, time = 0.0, last_dt = 1.0;
  int nplanes() const { return kp.nvm + 5; }
  size_t plane_bytes() const { return sizeof(double) * (size_t)kp.nc; }
};

#define CK(call)                                   \
  do {                                             \
    cudaError_t e__ = (call);                      \
    if (e__ != cudaSuccess) {                      \
      g_last_cuda_error = (int)e__;                \
      return PIP_ERR_CUDA;                         \
    }                                              \
  } while (0)

namespace {

// set_sym_mhd (Boundary_rot.f90:239-294), sign per ion variable for face f (0-based).
void sym_mhd(const pip_params &p, int f, signed char *out) {
  for (int n = 0; n < 9; ++n) out[n] = 1;
  const int dir = f / 2 + 1, b = p.flag_bnd[f];
  auto flip = [&](int var1) { out[var1 - 1] = -1; };  // 1-based variable number
  switch (b) {
    case 2: flip(1 + dir); flip(5 + dir); break;
    case 3: flip(1 + dir); flip(6 + dir % 3); flip(2 + (dir + 1) % 3); break;
    case 4: flip(1 + dir); flip(6 + (dir + 1) % 3); flip(2 + dir % 3); break;
    case 5: flip(1 + dir); flip(5 + dir); flip(2 + (dir + 1) % 3); flip(6 + (dir + 1) % 3); break;
    case 6: flip(1 + dir); flip(6 + dir % 3); flip(6 + (dir + 1) % 3); break;
    case 7: flip(2); flip(3); flip(4); break;
    default: break;
  }
  if (p.flag_divb == 1) {
    if (b == 2 || b == 20 || b == 5) out[8] = 1;
    else if (b == 3 || b == 4 || b == 6 || b == 7) out[8] = -1;
  }
}

// set_sym_hd (Boundary_rot.f90:296-320).
void sym_hd(const pip_params &p, int f, signed char *out) {
  for (int n = 0; n < 5; ++n) out[n] = 1;
  const int dir = f / 2 + 1, b = p.flag_bnd[f];
  auto flip = [&](int var1) { out[var1 - 1] = -1; };
  switch (b) {
    case 2: case 20: flip(1 + dir); break;
    case 3: flip(1 + dir); flip(2 + (dir + 1) % 3); break;
    case 4: flip(1 + dir); flip(2 + dir % 3); break;
    case 5: flip(1 + dir); flip(2 + (dir + 1) % 3); break;
    case 6: flip(1 + dir); break;
    default: break;
  }
}

// boundary_control type of a face code (MHDbnd/HDbnd, Boundary_rot.f90:62-80).
int bnd_type(int code) {
  switch (code) {
    case 3: case 4: case 5: case 6: case 7: case 11: return 2;
    default: return code;
  }
}

// Source index of ghost layer l on side s of an axis with n cells and m ghost layers
// (boundary_control's sr ranges, Boundary_rot.f90:338-368), 0-based.
int ghost_source(int type, int side, int l, int n, int m) {
  if (side == 0) {
    if (type == 1) return n - 2 * m + l;
    if (type == 2) return 2 * m - 1 - l;
    return m;  // type 10
  }
  if (type == 1) return m + l;
  if (type == 2) return n - m - 1 - l;
  return n - m - 1;
}

bool supported_bnd(int code) {
  switch (code) {
    case 1: case 2: case 3: case 4: case 5: case 6: case 7: case 10: case 11: return true;
    default: return false;
  }
}

int validate(const pip_params *p) {
  if (!p) return PIP_ERR_NULL;
  if (p->abi_version != PIP_ABI_VERSION) return PIP_ERR_PARAM;
  if (p->ndim != 1 && p->ndim != 2) return PIP_ERR_PARAM;
  if (p->kx != 1 || p->nvar_h != 5) return PIP_ERR_PARAM;
  if (p->ndim == 1 && p->flag_divb != 0) return PIP_ERR_PARAM;
  if (p->flag_divb != 0 && p->flag_divb != 1) return PIP_ERR_PARAM;
  if (p->nvar_m != (p->flag_divb == 1 ? 9 : 8)) return PIP_ERR_PARAM;
  if (p->flag_sch != 0 || p->flag_hll != 2 || p->s_order != 2 || p->t_order != 2 || p->flag_time != 0)
    return PIP_ERR_PARAM;
  // flag_col 1: constant alpha_c; 2..7: set_collisional col_type 1..6 (PIP_rot.f90:21-26),
  // per-cell alpha_c in the FP64 form, beta > 0 where alpha_c divides by sqrt(beta*gm/2)
  if (p->flag_col < 1 || p->flag_col > 7) return PIP_ERR_PARAM;
  if (p->flag_col >= 2 && p->precision != PIP_FP64) return PIP_ERR_PARAM;
  if ((p->flag_col == 2 || p->flag_col == 4 || p->flag_col == 6) && !(p->beta > 0.0))
    return PIP_ERR_PARAM;
  // flag_resi 1: a fixed eta field, 2: set_resistivity resi_type 2 or 3 at every stage (FP64
  // form); with conduction the margin would be 4
  if (p->flag_resi < 0 || p->flag_resi > 2) return PIP_ERR_PARAM;
  if (p->flag_resi >= 1 && (p->precision != PIP_FP64 || p->flag_heat != 0)) return PIP_ERR_PARAM;
  if (p->flag_resi == 2 && p->resi_type != 2 && p->resi_type != 3) return PIP_ERR_PARAM;
  if (p->flag_resi == 2 && p->resi_type == 3 && !(p->vd_cri > 0.0)) return PIP_ERR_PARAM;
  if (p->flag_pip_imp != 0 && p->flag_pip_imp != 1) return PIP_ERR_PARAM;
  if (p->flag_ir != PIP_IR_NONE && p->flag_ir != PIP_IR_POWERLAW && p->flag_ir != PIP_IR_POPESCU &&
      p->flag_ir != PIP_IR_POPESCU_EQ && p->flag_ir != PIP_IR_JEFFERY && p->flag_ir != PIP_IR_NLEVEL)
    return PIP_ERR_PARAM;
  if ((p->flag_ir == PIP_IR_POPESCU || p->flag_ir == PIP_IR_POPESCU_EQ ||
       p->flag_ir == PIP_IR_JEFFERY || p->flag_ir == PIP_IR_NLEVEL) &&
      (p->precision != PIP_FP64 || !(p->t_norm > 0.0) || !(p->n_norm > 0.0)))
    return PIP_ERR_PARAM;
  // flag_IR_type 0 (source_PIP's ionisation potential) exists for set_IR type 4 only: for the
  // other types the reference reads ion_pot and arb_heat before any call allocates them
  if (p->flag_ir != PIP_IR_NONE && p->flag_ir_type != 1 && p->flag_ir_type != 2 &&
      !(p->flag_ir == PIP_IR_NLEVEL && p->flag_ir_type == 0))
    return PIP_ERR_PARAM;
  if (p->flag_ir == PIP_IR_NLEVEL && p->flag_col % 2 == 0 && !(p->beta > 0.0)) return PIP_ERR_PARAM;
  if (p->precision != PIP_FP64 && p->precision != PIP_MIXED) return PIP_ERR_PARAM;
  if (p->flag_heat != 0 && p->flag_heat != 1) return PIP_ERR_PARAM;
  if (p->flag_heat == 1 && (p->ndim != 2 || p->hc_max < 0 || !(p->hc_error > 0.0) ||
                            !(p->kapper >= 0.0)))
    return PIP_ERR_PARAM;
  const int m0 = p->margin[0], m1 = p->margin[1];
  if (m0 < 2 || m0 > pip::kMaxMargin || p->margin[2] != 0) return PIP_ERR_PARAM;
  if (p->ndim == 1 && (m1 != 0 || p->jx != 1)) return PIP_ERR_PARAM;
  if (p->ndim == 2 && m1 != m0) return PIP_ERR_PARAM;
  if (p->ix - 2 * m0 < 4) return PIP_ERR_PARAM;
  if (p->ndim == 2 && p->jx - 2 * m1 < 4) return PIP_ERR_PARAM;
  for (int f = 0; f < 2 * p->ndim; ++f)
    if (!supported_bnd(p->flag_bnd[f])) return PIP_ERR_PARAM;
  if (!p->dx || !p->dy || !p->dz) return PIP_ERR_NULL;
  if (!(p->gm > 1.0) || !(p->safety > 0.0)) return PIP_ERR_PARAM;
  return PIP_OK;
}

// Constants of set_IR types 1-3 (PIP_rot.f90:134-228), with the Fortran's
// single-precision literals (2.7, 5.6e-16, 1.1604e4, 2.6e-19, 2.91e-14, 1.0e6) rounded to
// float first.
void ir_law_constants(const pip_params &p, KParams &k) {
  k.irs = (p.flag_ir == PIP_IR_POPESCU || p.flag_ir == PIP_IR_POPESCU_EQ ||
           p.flag_ir == PIP_IR_NLEVEL) ? p.flag_ir : 0;
  k.irf = p.flag_ir == PIP_IR_JEFFERY ? 1 : 0;
  k.irl = k.irs || k.irf ? 1 : 0;
  k.irn = p.flag_ir == PIP_IR_NLEVEL ? 1 : 0;
  if (k.irn) {
    // set_IR type 4 and IRgetionpot (PIP_rot.f90:232-296,1222-1233); tfac, the table and the
    // populations come with pip_set_nlevel
    k.nl_T0 = p.t_norm;
    k.nl_n0 = p.n_norm;
    k.nl_tir = p.t_ir;
    k.nl_odd = p.flag_col % 2 == 1 ? 1 : 0;
    k.nl_en_even = p.beta / p.t_norm / 2.0 / (double)8.6173e-5f;
    k.nl_lim = std::min(p.safety, 0.01);
    return;
  }
  if (k.irf) {
    // set_IR type 1 (PIP_rot.f90:135-149)
    const double T0 = p.t_norm, n0 = p.n_norm;
    k.ir_factor = std::exp(-13.2 / (T0 / 11605.0));
    const double f2 = (double)2.7f * std::pow(13.2 * 11605.0, -2.0) * std::pow(T0, 1.0 / 2.0) * n0;
    const double f3 = (double)5.6e-16f * std::pow(13.2 * 11605.0, -2.0) * std::pow(T0, -1.0) *
                      std::pow(n0, 2.0);
    k.ir_recfac = f2 / f3;
    k.ir_ionfac = f3 / p.t_ir;
    return;
  }
  if (!k.irs) return;
  const double te0 = p.t_norm / (double)1.1604e4f;
  const double n6 = p.n_norm * (double)1.0e6f;
  const double c26 = (double)2.6e-19f, c291 = (double)2.91e-14f;
  k.ir_c136 = 13.6 / te0;
  k.ir_n6 = n6;
  k.ir_c291 = c291;
  k.ir_c291n6 = c291 * n6;
  k.ir_tir = p.t_ir;
  if (k.irs == PIP_IR_POPESCU) {
    k.ir_recfac = c26 * n6 / std::sqrt(te0) * p.t_ir;
    return;
  }
  k.ir_recfac = c26 * n6 / std::sqrt(te0);
  const double ioneq = (c26 / std::sqrt(te0)) /
                       (c291 / (0.232 + 13.6 / te0) * std::pow(13.6 / te0, 0.39) * std::exp(-13.6 / te0));
  const double f_n = ioneq / (ioneq + 1.0), f_p = 1.0 - f_n;
  const double f_p_p = 2.0 * f_p / (f_n + 2.0 * f_p);
  k.ir_fp = f_p;
  k.ir_tfac = (p.flag_col % 2 == 1) ? 0.5 * f_p_p / f_p : p.beta / 2.0 * f_p_p * 5.0 / 6.0 / f_p;
  k.ir_sqtfac = std::sqrt(k.ir_tfac);
}

void build_kparams(pip_ctx *c) {
  const pip_params &p = c->p;
  KParams &k = c->kp;
  k.ndim = p.ndim;
  k.ix = p.ix;
  k.jx = p.jx;
  k.m0 = p.margin[0];
  k.m1 = p.ndim == 2 ? p.margin[1] : 0;
  k.nx = p.ix - 2 * k.m0;
  k.ny = p.ndim == 2 ? p.jx - 2 * k.m1 : 1;
  k.nvm = p.nvar_m;
  k.imp = p.flag_pip_imp;
  k.ir = p.flag_ir != PIP_IR_NONE;
  k.ir_type = p.flag_ir_type;
  ir_law_constants(p, k);
  k.nc = (long long)p.ix * p.jx;
  k.gm = p.gm;
  k.igm1 = 1.0 / (p.gm - 1.0);
  k.c32g = 3.0 / p.gm / 2.0;
  k.ro_lim = p.ro_lim;
  k.pr_lim = p.pr_lim;
  k.ac = p.col;
  k.safety = p.safety;
  double g = INFINITY;
  for (double v : c->dx) g = std::min(g, v);
  double gy = INFINITY, gz = INFINITY;
  for (double v : c->dy) gy = std::min(gy, v);
  for (double v : c->dz) gz = std::min(gz, v);
  k.sg_all = p.safety * std::min(std::min(g, gy), gz);
  k.col_lim = p.flag_pip_imp == 1 ? p.pip_imp_factor : std::min(p.safety, 0.3);
  k.ir_lim = std::min(p.safety, 0.1);
  k.ir_chi = p.ir_chi;
  k.ir_ion = p.ir_ion_coef;
  k.ir_rec = p.ir_rec_coef;
  // divb_cleaning_Dedner_source factor exp(-dt_sub/dt*safety*db_clean), dt_sub/dt = 1/2, 1
  k.decay[0] = std::exp(-0.5 * p.safety * p.db_clean);
  k.decay[1] = std::exp(-1.0 * p.safety * p.db_clean);
  k.dz0 = c->dz[0];
  k.hc_kapper = p.kapper;
  k.col_type = p.flag_col >= 2 ? p.flag_col - 1 : 0;
  k.resi = p.flag_resi;
  k.resi_dt = INFINITY;
  k.resi_type = p.resi_type;
  k.eta0 = p.eta_0;
  k.j_cri = p.j_cri;
  k.vd_cri = p.vd_cri;
  k.ac_b2g = p.beta / 2.0 * p.gm;
  k.ac_sb = std::sqrt(k.ac_b2g);
  for (int s = 0; s < 2; ++s) {
    const int fx = s, fy = 2 + s;
    k.typex[s] = bnd_type(p.flag_bnd[fx]);
    for (int l = 0; l < pip::kMaxMargin; ++l)
      k.gx[s][l] = l < k.m0 ? ghost_source(k.typex[s], s, l, p.ix, k.m0) : -1;
    signed char sm[9], sh[5];
    sym_mhd(p, fx, sm);
    sym_hd(p, fx, sh);
    for (int n = 0; n < k.nvm; ++n) k.symx[s][n] = sm[n];
    for (int n = 0; n < 5; ++n) k.symx[s][k.nvm + n] = sh[n];
    if (p.ndim == 2) {
      k.typey[s] = bnd_type(p.flag_bnd[fy]);
      for (int l = 0; l < pip::kMaxMargin; ++l)
        k.gy[s][l] = l < k.m1 ? ghost_source(k.typey[s], s, l, p.jx, k.m1) : -1;
      sym_mhd(p, fy, sm);
      sym_hd(p, fy, sh);
      for (int n = 0; n < k.nvm; ++n) k.symy[s][n] = sm[n];
      for (int n = 0; n < 5; ++n) k.symy[s][k.nvm + n] = sh[n];
    } else {
      k.typey[s] = 1;
      for (int l = 0; l < pip::kMaxMargin; ++l) k.gy[s][l] = -1;
      for (int n = 0; n < pip::kMaxPlanes; ++n) k.symy[s][n] = 1;
    }
  }
}

}  // namespace

void pip::record_cuda_error(int code) { g_last_cuda_error = code; }

// Kernel parameters straight from a parameter block, for callers without a context: the
// same validation and tables as pip_ctx_create, built on the stack (no allocation).  The
// dx/dy pointers of the result are left null for the caller to point at device copies.
int pip::kparams_from_params(const pip_params *p, KParams *k) {
  const int st = validate(p);
  if (st != PIP_OK) return st;
  // the per-cell alpha_c and eta fields and the per-stage rates live in a context
  if (p->flag_col != 1 || p->flag_resi != 0) return PIP_ERR_PARAM;
  if (p->flag_ir != PIP_IR_NONE && p->flag_ir != PIP_IR_POWERLAW) return PIP_ERR_PARAM;
  *k = KParams{};
  k->resi_dt = INFINITY;
  k->ndim = p->ndim;
  k->ix = p->ix;
  k->jx = p->jx;
  k->m0 = p->margin[0];
  k->m1 = p->ndim == 2 ? p->margin[1] : 0;
  k->nx = p->ix - 2 * k->m0;
  k->ny = p->ndim == 2 ? p->jx - 2 * k->m1 : 1;
  k->nvm = p->nvar_m;
  k->imp = p->flag_pip_imp;
  k->ir = p->flag_ir != PIP_IR_NONE;
  k->ir_type = p->flag_ir_type;
  k->nc = (long long)p->ix * p->jx;
  k->gm = p->gm;
  k->igm1 = 1.0 / (p->gm - 1.0);
  k->c32g = 3.0 / p->gm / 2.0;
  k->ro_lim = p->ro_lim;
  k->pr_lim = p->pr_lim;
  k->ac = p->col;
  k->safety = p->safety;
  double g = INFINITY, gy = INFINITY, gz = INFINITY;
  for (int i = 0; i < p->ix; ++i) g = std::min(g, p->dx[i]);
  for (int j = 0; j < p->jx; ++j) gy = std::min(gy, p->dy[j]);
  for (int q = 0; q < p->kx; ++q) gz = std::min(gz, p->dz[q]);
  k->sg_all = p->safety * std::min(std::min(g, gy), gz);
  k->col_lim = p->flag_pip_imp == 1 ? p->pip_imp_factor : std::min(p->safety, 0.3);
  k->ir_lim = std::min(p->safety, 0.1);
  k->ir_chi = p->ir_chi;
  k->ir_ion = p->ir_ion_coef;
  k->ir_rec = p->ir_rec_coef;
  k->decay[0] = std::exp(-0.5 * p->safety * p->db_clean);
  k->decay[1] = std::exp(-1.0 * p->safety * p->db_clean);
  k->dz0 = p->dz[0];
  k->hc_kapper = p->kapper;
  for (int s = 0; s < 2; ++s) {
    k->typex[s] = bnd_type(p->flag_bnd[s]);
    for (int l = 0; l < pip::kMaxMargin; ++l)
      k->gx[s][l] = l < k->m0 ? ghost_source(k->typex[s], s, l, p->ix, k->m0) : -1;
    signed char sm[9], sh[5];
    sym_mhd(*p, s, sm);
    sym_hd(*p, s, sh);
    for (int n = 0; n < k->nvm; ++n) k->symx[s][n] = sm[n];
    for (int n = 0; n < 5; ++n) k->symx[s][k->nvm + n] = sh[n];
    if (p->ndim == 2) {
      k->typey[s] = bnd_type(p->flag_bnd[2 + s]);
      for (int l = 0; l < pip::kMaxMargin; ++l)
        k->gy[s][l] = l < k->m1 ? ghost_source(k->typey[s], s, l, p->jx, k->m1) : -1;
      sym_mhd(*p, 2 + s, sm);
      sym_hd(*p, 2 + s, sh);
      for (int n = 0; n < k->nvm; ++n) k->symy[s][n] = sm[n];
      for (int n = 0; n < 5; ++n) k->symy[s][k->nvm + n] = sh[n];
    } else {
      k->typey[s] = 1;
      for (int l = 0; l < pip::kMaxMargin; ++l) k->gy[s][l] = -1;
      for (int n = 0; n < pip::kMaxPlanes; ++n) k->symy[s][n] = 1;
    }
  }
  return PIP_OK;
}

namespace {

// Host copy of the device finalize_dt (same IEEE operations, same order).
double finalize_dt_host(const KParams &k, const DevCtrl &c, int slot) {
  double dt, rho, gr;
  std::memcpy(&dt, &c.red_dt[slot], sizeof(double));
  std::memcpy(&rho, &c.red_rho[slot], sizeof(double));
  std::memcpy(&gr, &c.red_gr[slot], sizeof(double));
  dt = std::fmin(dt, k.col_lim / rho);
  if (k.ir) dt = std::fmin(dt, k.ir_lim / std::fmax(gr, 1.0e-5));
  if (k.irn) {
    double ip, nx;
    std::memcpy(&ip, &c.red_ip[slot], sizeof(double));
    std::memcpy(&nx, &c.red_nx[slot], sizeof(double));
    if (k.ir_type == 0) dt = std::fmin(dt, k.safety / ip);
    dt = std::fmin(dt, k.nl_lim / nx);
  }
  return dt;
}

// A reduction slot before a cfl: the min-CFL candidate starts at cfl_mhd's 10.0 and
// cfl_resi's bound (min is exact and commutative, so the order of the terms is free).
void reset_slot(DevCtrl &h, int slot, const KParams &k) {
  const double seed = std::fmin(10.0, k.resi_dt);
  std::memcpy(&h.red_dt[slot], &seed, sizeof(double));
  h.red_rho[slot] = 0ull;
  h.red_gr[slot] = 0ull;
  h.red_ip[slot] = 0ull;
  h.red_nx[slot] = 0ull;
}

// cfl_resi (Scheme_rot.f90:291-302) for a fixed eta field: the minimum over the interior
// cells of safety*gmin**2/max(eta,1e-8), gmin = min(dx(i),dy(j),dz(1)).
double resi_bound(const pip_ctx *c, const double *eta) {
  const KParams &k = c->kp;
  double dt = INFINITY;
  for (int j = k.m1; j < k.jx - k.m1; ++j)
    for (int i = k.m0; i < k.ix - k.m0; ++i) {
      const double gmin = std::fmin(std::fmin(c->dx[i], c->dy[j]), c->dz[0]);
      dt = std::fmin(dt, c->p.safety * (gmin * gmin) / std::fmax(eta[(size_t)j * k.ix + i], 1.0e-8));
    }
  return dt;
}

int sync_ctrl_to_host(pip_ctx *c) {
  CK(cudaMemcpyAsync(c->h_ctrl, c->ctrl, sizeof(DevCtrl), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PIP_OK;
}

// The control fields a host-stepped stage reads, set on the device from launch arguments
// (no pinned host buffer that a later call could rewrite before the copy runs).
__global__ void stage_ctrl_kernel(DevCtrl *ctrl, double dt, double cmax) {
  ctrl->dt = dt;
  ctrl->cmax = cmax;
  ctrl->done = 0;
  ctrl->nan_flag = 0;
  ctrl->status = 0;
  ctrl->blocks_done = 0;
}

// set_coefficients(U_h,U_m,0) of the prologue (Initial_rot.f90:140) for a state uploaded
// since the last one: set_collisional (alpha_c per cell) and set_IR (types 1-3) rewrite the
// energies and set their fields before the first cfl and the first stage.
int ensure_coefficients(pip_ctx *c) {
  if ((!c->kp.col_type && !c->kp.irl && c->kp.resi != 2) || c->coef_valid) return PIP_OK;
  if (c->kp.irn) {
    // set_IR type 4 inside set_coefficients: on a fresh start first its reference block
    // (Gm_rec_ref, the initial ion_pot), then the rates of the state; before the energy
    // rewrites of coefficients_kernel, whose sequence the rates kernel repeats on its copies
    int ipmode = 0;
    if (!c->nl_init) {
      CK(c->L->nlev_ref(c->kp, c->nl_ref, c->stream));
      double gref = 0.0;
      CK(cudaMemcpyAsync(&gref, c->nl_ref + 36, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      c->kp.nl_gref = gref;
      c->nl_init = true;
      ipmode = c->kp.ir_type == 0 ? 2 : 0;
    }
    CK(c->L->nlev_rates(c->kp, c->A, c->kp.col_type ? 1 : 0, ipmode, c->nl_ref, c->ctrl, c->stream));
  }
  CK(c->L->coefficients(c->kp, c->A, c->stream));
  c->coef_valid = true;
  return PIP_OK;
}

// set_IR type 4 needs pip_set_nlevel first.
bool nl_missing(const pip_ctx *c) { return c->kp.irn && !c->nl_ready; }

// Nexcite's update target becomes the current set.
void nl_swap(pip_ctx *c) {
  c->nl_cur ^= 1;
  c->kp.nl_nex = c->nl_nex[c->nl_cur];
  c->kp.nl_nex2 = c->nl_nex[c->nl_cur ^ 1];
}

int push_ctrl(pip_ctx *c) {
  CK(cudaMemcpyAsync(c->ctrl, c->h_ctrl, sizeof(DevCtrl), cudaMemcpyHostToDevice, c->stream));
  return PIP_OK;
}

// One RK stage of the context's precision form (rows: every tile row, or the first and
// last / the middle ones, see Launchers::stage).
cudaError_t do_stage(pip_ctx *c, int stage, int dt_mode, int epi, int rows = 0) {
  if (c->mixed) {
    if (stage == 1)
      return pip::mixed_stage(c->kp, 1, c->Ahi, c->Ahi, nullptr, c->Bf, nullptr, c->ctrl, dt_mode,
                              epi, c->stream, c->tma ? &c->tm_a : nullptr, rows);
    return pip::mixed_stage(c->kp, 2, c->Bf, c->Ahi, c->Alo, c->Ahi, c->Alo, c->ctrl, dt_mode, epi,
                            c->stream, c->tma ? &c->tm_b : nullptr, rows);
  }
  if (c->kp.irn) {
    // set_IR type 4 of the stage (set_coefficients, after set_collisional's rewrite), the
    // stage, then hydrogen_excitation_update on the updated state (Solver_rot.f90:218-220)
    const double *Us = stage == 1 ? c->A : c->B;
    double *Uo = stage == 1 ? c->B : c->A;
    cudaError_t e = c->L->nlev_rates(c->kp, Us, c->kp.col_type ? 1 : 0, c->kp.ir_type == 0 ? 1 : 0,
                                     nullptr, c->ctrl, c->stream);
    if (e != cudaSuccess) return e;
    e = c->L->stage(c->kp, stage, Us, c->A, Uo, c->ctrl, dt_mode, epi, c->stream,
                    c->tma ? (stage == 1 ? &c->tm_a : &c->tm_b) : nullptr, rows);
    if (e != cudaSuccess) return e;
    e = c->L->nlev_update(c->kp, Uo, c->ctrl, stage, c->stream);
    if (e == cudaSuccess) nl_swap(c);
    return e;
  }
  if (stage == 1)
    return c->L->stage(c->kp, 1, c->A, c->A, c->B, c->ctrl, dt_mode, epi, c->stream,
                       c->tma ? &c->tm_a : nullptr, rows);
  return c->L->stage(c->kp, 2, c->B, c->A, c->A, c->ctrl, dt_mode, epi, c->stream,
                     c->tma ? &c->tm_b : nullptr, rows);
}

cudaError_t do_cfl(pip_ctx *c, int slot) {
  if (c->mixed) return pip::mixed_cfl(c->kp, c->Ahi, c->Alo, c->ctrl, slot, c->stream);
  if (c->kp.irn) {
    // the time loop's set_IR before the cfl, the cfl, then its type-4 terms
    cudaError_t e = c->L->nlev_rates(c->kp, c->A, 0, 0, nullptr, c->ctrl, c->stream);
    if (e != cudaSuccess) return e;
    if ((e = c->L->cfl(c->kp, c->A, c->ctrl, slot, c->stream)) != cudaSuccess) return e;
    return c->L->nlev_cfl(c->kp, c->A, c->ctrl, slot, c->stream);
  }
  return c->L->cfl(c->kp, c->A, c->ctrl, slot, c->stream);
}

// The mixed form keeps its state in (hi, lo); these move it through the FP64 array A.
cudaError_t to_fp64(pip_ctx *c) {
  if (!c->mixed) return cudaSuccess;
  return pip::mixed_join(c->Ahi, c->Alo, c->A, c->kp.nc * c->nplanes(), c->stream);
}
cudaError_t from_fp64(pip_ctx *c) {
  if (!c->mixed) return cudaSuccess;
  return pip::mixed_split(c->A, c->Ahi, c->Alo, c->kp.nc * c->nplanes(), c->stream);
}

// post_step's implicit conduction (Solver_rot.f90:296-303) on the context state with the dt
// at dtp (device) and the ghost fill that follows it in run_solver (:78).
int conduct(pip_ctx *c, const double *dtp, int *iters, double *relres, int *status) {
  CK(to_fp64(c));
  CK(pip::hc_run(c->hc, c->kp, c->A, dtp, c->p.hc_error, c->p.hc_max, c->stream, iters, relres,
                 status));
  CK(c->L->ghosts(c->kp, c->A, c->stream));
  CK(from_fp64(c));
  return PIP_OK;
}

// K steps of [stage 1, stage 2] as launched by pip_run.
int launch_steps(pip_ctx *c, int k) {
  for (int s = 0; s < k; ++s) {
    cudaError_t e = do_stage(c, 1, 1, 0);
    if (e == cudaSuccess) e = do_stage(c, 2, 1, -1);
    if (e != cudaSuccess) {
      g_last_cuda_error = (int)e;
      return PIP_ERR_CUDA;
    }
  }
  return PIP_OK;
}

int ensure_graph(pip_ctx *c, int k) {
  if (c->graph && c->graph_steps == k) return PIP_OK;
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int st = launch_steps(c, k);
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (st != PIP_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  CK(e);
  e = cudaGraphInstantiate(&c->graph, g, 0);
  cudaGraphDestroy(g);
  CK(e);
  c->graph_steps = k;
  return PIP_OK;
}

int ensure_scratch(pip_ctx *c) {
  if (!c->scratch) CK(cudaMalloc(&c->scratch, c->plane_bytes() * c->nplanes()));
  return PIP_OK;
}

int set_device(pip_ctx *c) {
  CK(cudaSetDevice(c->device));
  return PIP_OK;
}

}  // namespace

extern "C" {

int pip_ctx_create(const pip_params *p, pip_ctx **out) {
  if (!out) return PIP_ERR_NULL;
  *out = nullptr;
  int st = validate(p);
  if (st != PIP_OK) return st;
  pip_ctx *c = new (std::nothrow) pip_ctx();
  if (!c) return PIP_ERR_NOMEM;
  c->p = *p;
  c->dx.assign(p->dx, p->dx + p->ix);
  c->dy.assign(p->dy, p->dy + p->jx);
  c->dz.assign(p->dz, p->dz + p->kx);
  c->p.dx = c->p.dy = c->p.dz = nullptr;
  build_kparams(c);
  c->L = p->fp_exact ? &pip::launchers_exact() : &pip::launchers_fast();
  c->mixed = p->precision == PIP_MIXED;
  auto fail = [&](cudaError_t e) {
    g_last_cuda_error = (int)e;
    pip_ctx_destroy(c);
    return e == cudaErrorMemoryAllocation ? PIP_ERR_NOMEM : PIP_ERR_CUDA;
  };
  cudaError_t e = cudaGetDevice(&c->device);
  if (e != cudaSuccess) return fail(e);
  if ((e = c->L->prepare()) != cudaSuccess) return fail(e);
  if (c->mixed && (e = pip::mixed_prepare()) != cudaSuccess) return fail(e);
  if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
  const size_t state = c->plane_bytes() * c->nplanes();
  if ((e = cudaMalloc(&c->A, state)) != cudaSuccess) return fail(e);
  if (c->mixed) {
    const size_t fstate = state / 2;
    if ((e = cudaMalloc(&c->Ahi, fstate)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&c->Alo, fstate)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&c->Bf, fstate)) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(c->Bf, 0, fstate)) != cudaSuccess) return fail(e);
    // 2D tiles of the stage sources by TMA where the grid meets its alignment rules
    c->tma = pip::mixed_tile_map(c->kp, c->Ahi, &c->tm_a) &&
             pip::mixed_tile_map(c->kp, c->Bf, &c->tm_b);
  } else if ((e = cudaMalloc(&c->B, state)) != cudaSuccess) {
    return fail(e);
  } else {
    c->tma = c->L->tile_map(c->kp, c->A, &c->tm_a) && c->L->tile_map(c->kp, c->B, &c->tm_b);
  }
  if ((e = cudaMalloc(&c->d_dx, sizeof(double) * p->ix)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&c->d_dy, sizeof(double) * p->jx)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&c->ctrl, sizeof(DevCtrl))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&c->d_flag, sizeof(int))) != cudaSuccess) return fail(e);
  if ((e = cudaMallocHost(&c->h_ctrl, sizeof(DevCtrl))) != cudaSuccess) return fail(e);
  std::memset(c->h_ctrl, 0, sizeof(DevCtrl));
  if ((e = cudaMemcpy(c->d_dx, c->dx.data(), sizeof(double) * p->ix, cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(e);
  if ((e = cudaMemcpy(c->d_dy, c->dy.data(), sizeof(double) * p->jx, cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(e);
  if ((e = cudaMemset(c->A, 0, state)) != cudaSuccess) return fail(e);
  if (c->B && (e = cudaMemset(c->B, 0, state)) != cudaSuccess) return fail(e);
  if ((e = cudaMemcpy(c->ctrl, c->h_ctrl, sizeof(DevCtrl), cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(e);
  c->kp.dx = c->d_dx;
  c->kp.dy = c->d_dy;
  if ((e = cudaMalloc(&c->d_dt, sizeof(double))) != cudaSuccess) return fail(e);
  if (c->kp.resi == 2) {
    // eta follows the state: the bound of the eta of the last set_resistivity
    if ((e = cudaMalloc(&c->d_resi, sizeof(unsigned long long))) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(c->d_resi, 0, sizeof(unsigned long long))) != cudaSuccess) return fail(e);
    c->kp.resi_bound = c->d_resi;
  } else if (c->kp.resi) {
    // set_resistivity type 0 until pip_set_resistivity gives another field
    std::vector<double> eta((size_t)c->kp.nc, p->eta_0);
    if ((e = cudaMalloc(&c->etaf, c->plane_bytes())) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpy(c->etaf, eta.data(), c->plane_bytes(), cudaMemcpyHostToDevice)) != cudaSuccess)
      return fail(e);
    c->kp.etaf = c->etaf;
    c->kp.resi_dt = resi_bound(c, eta.data());
  }
  if (c->kp.irn) {
    for (int k = 0; k < 2; ++k) {
      if ((e = cudaMalloc(&c->nl_nex[k], 6 * c->plane_bytes())) != cudaSuccess) return fail(e);
      if ((e = cudaMemset(c->nl_nex[k], 0, 6 * c->plane_bytes())) != cudaSuccess) return fail(e);
    }
    if ((e = cudaMalloc(&c->nl_cr, 36 * c->plane_bytes())) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(c->nl_cr, 0, 36 * c->plane_bytes())) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&c->nl_ip, c->plane_bytes())) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(c->nl_ip, 0, c->plane_bytes())) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&c->nl_ref, 37 * sizeof(double))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&c->nl_k, sizeof(pip::NlevConst))) != cudaSuccess) return fail(e);
    c->kp.nl_nex = c->nl_nex[0];
    c->kp.nl_nex2 = c->nl_nex[1];
    c->kp.nl_cr = c->nl_cr;
    c->kp.nl_ip = c->nl_ip;
    c->kp.nl_k = c->nl_k;
  }
  if (c->kp.irf || c->kp.irn) {
    if ((e = cudaMalloc(&c->irg, 2 * c->plane_bytes())) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(c->irg, 0, 2 * c->plane_bytes())) != cudaSuccess) return fail(e);
    c->kp.irg = c->irg;
  }
  if (c->kp.col_type) {
    if ((e = cudaMalloc(&c->acf, c->plane_bytes())) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(c->acf, 0, c->plane_bytes())) != cudaSuccess) return fail(e);
    c->kp.acf = c->acf;
  }
  if (p->flag_heat == 1 && (e = pip::hc_create(c->kp, c->mixed, &c->hc)) != cudaSuccess)
    return fail(e);
  if (c->mixed) {
    std::vector<double> r(c->dx.size()), ry(c->dy.size());
    for (size_t i = 0; i < r.size(); ++i) r[i] = 1.0 / c->dx[i];
    for (size_t j = 0; j < ry.size(); ++j) ry[j] = 1.0 / c->dy[j];
    if ((e = cudaMalloc(&c->d_rdx, sizeof(double) * r.size())) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&c->d_rdy, sizeof(double) * ry.size())) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpy(c->d_rdx, r.data(), sizeof(double) * r.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
      return fail(e);
    if ((e = cudaMemcpy(c->d_rdy, ry.data(), sizeof(double) * ry.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
      return fail(e);
    c->kp.rdx = c->d_rdx;
    c->kp.rdy = c->d_rdy;
  }
  *out = c;
  return PIP_OK;
}

void pip_ctx_destroy(pip_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->graph) cudaGraphExecDestroy(c->graph);
  cudaFree(c->A);
  cudaFree(c->B);
  cudaFree(c->Ahi);
  cudaFree(c->Alo);
  cudaFree(c->Bf);
  cudaFree(c->d_dx);
  cudaFree(c->d_dy);
  cudaFree(c->d_rdx);
  cudaFree(c->d_rdy);
  cudaFree(c->scratch);
  cudaFree(c->ctrl);
  cudaFree(c->d_flag);
  cudaFree(c->d_dt);
  cudaFree(c->acf);
  cudaFree(c->etaf);
  cudaFree(c->d_resi);
  if (c->rows_stream) cudaStreamDestroy(c->rows_stream);
  for (cudaEvent_t ev : c->rows_ev)
    if (ev) cudaEventDestroy(ev);
  cudaFree(c->irg);
  cudaFree(c->nl_nex[0]);
  cudaFree(c->nl_nex[1]);
  cudaFree(c->nl_cr);
  cudaFree(c->nl_ip);
  cudaFree(c->nl_tab);
  cudaFree(c->nl_ref);
  cudaFree(c->nl_k);
  cudaFree(c->nl_rtab);
  pip::hc_destroy(c->hc);
  if (c->h_ctrl) cudaFreeHost(c->h_ctrl);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int pip_upload(pip_ctx *c, const double *U_h, const double *U_m) {
  if (!c || !U_h || !U_m) return PIP_ERR_NULL;
  c->dev_loop = false;
  if (set_device(c)) return PIP_ERR_CUDA;
  const size_t pb = c->plane_bytes();
  CK(cudaMemcpyAsync(c->A, U_m, pb * c->kp.nvm, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->A + (size_t)c->kp.nvm * c->kp.nc, U_h, pb * 5, cudaMemcpyHostToDevice, c->stream));
  CK(from_fp64(c));
  CK(cudaStreamSynchronize(c->stream));
  c->uploaded = true;
  c->coef_valid = false;
  c->last_stage = 0;
  return PIP_OK;
}

int pip_download(pip_ctx *c, double *U_h, double *U_m) {
  if (!c || !U_h || !U_m) return PIP_ERR_NULL;
  if (!c->uploaded) return PIP_ERR_STATE;
  if (set_device(c)) return PIP_ERR_CUDA;
  const size_t pb = c->plane_bytes();
  CK(to_fp64(c));
  CK(cudaMemcpyAsync(U_m, c->A, pb * c->kp.nvm, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(U_h, c->A + (size_t)c->kp.nvm * c->kp.nc, pb * 5, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PIP_OK;
}

int pip_cfl(pip_ctx *c, double *dt, double *cmax) {
  if (!c) return PIP_ERR_NULL;
  if (!c->uploaded || nl_missing(c)) return PIP_ERR_STATE;
  if (set_device(c)) return PIP_ERR_CUDA;
  if (ensure_coefficients(c)) return PIP_ERR_CUDA;
  reset_slot(*c->h_ctrl, 0, c->kp);
  c->h_ctrl->status = 0;
  if (push_ctrl(c)) return PIP_ERR_CUDA;
  CK(do_cfl(c, 0));
  if (sync_ctrl_to_host(c)) return PIP_ERR_CUDA;
  if (c->h_ctrl->status) return c->h_ctrl->status;
  const double d = finalize_dt_host(c->kp, *c->h_ctrl, 0);
  c->dt = d;
  if (c->p.flag_divb >= 1) c->cmax = c->kp.sg_all / d;
  if (dt) *dt = d;
  if (cmax) *cmax = c->cmax;
  return PIP_OK;
}

int pip_step(pip_ctx *c, double dt) {
  if (!c) return PIP_ERR_NULL;
  if (!c->uploaded || c->exchanged || nl_missing(c)) return PIP_ERR_STATE;
  if (!(dt > 0.0) || !std::isfinite(dt)) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  if (ensure_coefficients(c)) return PIP_ERR_CUDA;
  DevCtrl &h = *c->h_ctrl;
  h.dt = dt;
  h.cmax = c->cmax;
  h.done = 0;
  h.nan_flag = 0;
  h.status = 0;
  h.blocks_done = 0;
  if (push_ctrl(c)) return PIP_ERR_CUDA;
  CK(do_stage(c, 1, 0, 0));
  CK(do_stage(c, 2, 0, 0));
  if (c->hc) {
    CK(cudaMemcpyAsync(c->d_dt, &c->h_ctrl->dt, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    int it = 0, st = 0;
    const int r = conduct(c, c->d_dt, &it, nullptr, &st);
    if (r != PIP_OK) return r;
    c->hc_iters = it;
  }
  CK(cudaStreamSynchronize(c->stream));
  c->last_dt = dt;
  c->last_stage = 2;
  if (c->kp.irn) {   // a negative rate of the 6-level model
    if (sync_ctrl_to_host(c)) return PIP_ERR_CUDA;
    if (h.status) return h.status;
  }
  return PIP_OK;
}

static int run_loop(pip_ctx *c, int64_t nsteps, double t_end, double *time_out,
                    int64_t *steps_done, float *device_ms) {
  if (!c) return PIP_ERR_NULL;
  if (!c->uploaded || c->exchanged || nl_missing(c)) return PIP_ERR_STATE;
  if (nsteps <= 0 && !(t_end > 0.0)) return PIP_ERR_PARAM;
  c->last_stage = 2;
  c->dev_loop = false;
  if (set_device(c)) return PIP_ERR_CUDA;
  if (ensure_coefficients(c)) return PIP_ERR_CUDA;
  if ((t_end > 0.0 && c->time >= t_end)) {
    if (time_out) *time_out = c->time;
    if (steps_done) *steps_done = 0;
    return PIP_OK;
  }
  DevCtrl &h = *c->h_ctrl;
  std::memset(&h, 0, sizeof(DevCtrl));
  h.time = c->time;
  h.t_end = t_end > 0.0 ? t_end : 0.0;
  h.nsteps = nsteps > 0 ? nsteps : 0;
  h.cmax = c->cmax;
  reset_slot(h, 0, c->kp);
  reset_slot(h, 1, c->kp);
  if (push_ctrl(c)) return PIP_ERR_CUDA;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (device_ms) {
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    if (nsteps > 0 && !(t_end > 0.0) && nsteps >= 32) {
      int st0 = ensure_graph(c, 32);  // instantiate before the timed region
      if (st0 != PIP_OK) return st0;
    }
    CK(cudaEventRecord(ev0, c->stream));
  }
  // cfl of the first step (main.f90:36); later steps get it fused into stage 2
  CK(do_cfl(c, 0));
  bool halted = false;
  if (c->kp.irn) {
    // a negative rate of the 6-level model stops the run before the step, as
    // get_col_ion_coeff stops the program inside set_IR
    if (sync_ctrl_to_host(c)) return PIP_ERR_CUDA;
    halted = h.status != 0;
  }
  if (c->hc || c->kp.resi == 2 || c->kp.irn) {
    // conduction runs: the stages, post_step's conduction and the ghost fill, then the two
    // cfl calls (rewrite; rewrite + next dt) as separate kernels; the host loop waits on
    // BiCGstab's convergence checks anyway, so no graph.  Per-stage eta: whether a step
    // was the last is known only once stage 2 has lowered its time increment to cfl_resi's
    // bound, so the next cfl's rewrite cannot be fused into stage 2 either.  set_IR type 4:
    // the rates, excitation-update and cfl kernels of the 6-level model sit between the
    // stages and the cfl calls.
    long long n = 0;
    int total_it = 0;
    while (!halted) {
      CK(do_stage(c, 1, 1, 0));
      CK(do_stage(c, 2, 1, 0));
      if (c->hc) {
        int it = 0, hst = 0;
        const int r = conduct(c, &c->ctrl->dt, &it, nullptr, &hst);
        if (r != PIP_OK) return r;
        total_it += it;
      }
      if (sync_ctrl_to_host(c)) return PIP_ERR_CUDA;
      if (h.nan_flag || h.status || h.step != n + 1) break;
      CK(do_cfl(c, (int)(n & 1)));          // the cfl after run_solver (main.f90:47)
      if (h.done) break;
      CK(do_cfl(c, (int)((n + 1) & 1)));    // the next step's cfl (main.f90:36)
      ++n;
      if (c->kp.irn) {
        if (sync_ctrl_to_host(c)) return PIP_ERR_CUDA;
        if (h.status) break;
      }
    }
    c->hc_iters = total_it;
    if (device_ms) {
      CK(cudaEventRecord(ev1, c->stream));
      CK(cudaEventSynchronize(ev1));
    }
  } else {
  const int K = 32;
  int st = PIP_OK;
  if (nsteps > 0 && !(t_end > 0.0)) {
    // known step count: whole graphs, then the remainder launched directly
    int64_t left = nsteps;
    if (left >= K) {
      if ((st = ensure_graph(c, K)) != PIP_OK) return st;
      for (; left >= K; left -= K) CK(cudaGraphLaunch(c->graph, c->stream));
    }
    if (left > 0 && (st = launch_steps(c, (int)left)) != PIP_OK) return st;
    if (device_ms) CK(cudaEventRecord(ev1, c->stream));
    if (sync_ctrl_to_host(c)) return PIP_ERR_CUDA;
  } else {
    if ((st = ensure_graph(c, K)) != PIP_OK) return st;
    for (;;) {
      CK(cudaGraphLaunch(c->graph, c->stream));
      if (sync_ctrl_to_host(c)) return PIP_ERR_CUDA;
      if (h.done || h.nan_flag) break;
    }
    if (device_ms) {
      CK(cudaEventRecord(ev1, c->stream));
      CK(cudaEventSynchronize(ev1));
    }
  }
  }
  if (device_ms) {
    CK(cudaEventElapsedTime(device_ms, ev0, ev1));
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
  }
  c->time = h.time;
  c->dt = h.dt;
  c->last_dt = h.dt;
  c->cmax = h.cmax;
  if (time_out) *time_out = h.time;
  if (steps_done) *steps_done = h.step;
  if (h.status == PIP_ERR_RATE) return PIP_ERR_RATE;
  if (h.nan_flag) return PIP_ERR_NAN;
  if (h.status) return h.status;
  return PIP_OK;
}

int pip_run(pip_ctx *c, int64_t nsteps, double t_end, double *time_out, int64_t *steps_done) {
  return run_loop(c, nsteps, t_end, time_out, steps_done, nullptr);
}

int pip_run_timed(pip_ctx *c, int64_t nsteps, double t_end, double *time_out,
                  int64_t *steps_done, float *device_ms) {
  if (!device_ms) return PIP_ERR_NULL;
  return run_loop(c, nsteps, t_end, time_out, steps_done, device_ms);
}

int pip_bench_stage_ms(pip_ctx *c, int nsteps, float *ms1, float *ms2, float *msstep) {
  if (!c || !ms1 || !ms2 || !msstep) return PIP_ERR_NULL;
  if (!c->uploaded) return PIP_ERR_STATE;
  if (nsteps <= 0 || c->kp.irn) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  DevCtrl &h = *c->h_ctrl;
  std::memset(&h, 0, sizeof(DevCtrl));
  h.time = c->time;
  h.nsteps = nsteps;
  reset_slot(h, 0, c->kp);
  reset_slot(h, 1, c->kp);
  if (ensure_coefficients(c)) return PIP_ERR_CUDA;
  if (push_ctrl(c)) return PIP_ERR_CUDA;
  CK(do_cfl(c, 0));
  std::vector<cudaEvent_t> ev(3 * (size_t)nsteps);
  for (auto &e : ev) CK(cudaEventCreate(&e));
  for (int s = 0; s < nsteps; ++s) {
    CK(cudaEventRecord(ev[3 * s], c->stream));
    CK(do_stage(c, 1, 1, 0));
    CK(cudaEventRecord(ev[3 * s + 1], c->stream));
    CK(do_stage(c, 2, 1, -1));
    CK(cudaEventRecord(ev[3 * s + 2], c->stream));
  }
  if (sync_ctrl_to_host(c)) return PIP_ERR_CUDA;
  double t1 = 0.0, t2 = 0.0;
  for (int s = 0; s < nsteps; ++s) {
    float a = 0.f, b = 0.f;
    CK(cudaEventElapsedTime(&a, ev[3 * s], ev[3 * s + 1]));
    CK(cudaEventElapsedTime(&b, ev[3 * s + 1], ev[3 * s + 2]));
    t1 += a;
    t2 += b;
  }
  for (auto &e : ev) cudaEventDestroy(e);
  c->time = h.time;
  *ms1 = (float)(t1 / nsteps);
  *ms2 = (float)(t2 / nsteps);
  *msstep = (float)((t1 + t2) / nsteps);
  return PIP_OK;
}

int64_t pip_kernels_per_run(pip_ctx *c, int64_t nsteps) {
  const int64_t init = c && (c->kp.col_type || c->kp.irl) && !c->coef_valid ? 1 : 0;  // set_coefficients(0)
  return init + 1 + 2 * (nsteps > 0 ? nsteps : 0);
}

int64_t pip_conduction_iterations(pip_ctx *c) { return c ? c->hc_iters : 0; }

int pip_set_time(pip_ctx *c, double t) {
  if (!c) return PIP_ERR_NULL;
  c->time = t;
  return PIP_OK;
}

int pip_get_time(pip_ctx *c, double *t) {
  if (!c || !t) return PIP_ERR_NULL;
  *t = c->time;
  return PIP_OK;
}

int pip_flux(pip_ctx *c, int dir, double *F_h, double *F_m) {
  if (!c || !F_h || !F_m) return PIP_ERR_NULL;
  if (!c->uploaded) return PIP_ERR_STATE;
  if (dir < 1 || dir > c->kp.ndim) return PIP_ERR_PARAM;
  if (c->mixed) return PIP_ERR_STATE;  // unit-level entry points are FP64 only
  if (set_device(c) || ensure_scratch(c) || ensure_coefficients(c)) return PIP_ERR_CUDA;
  const size_t pb = c->plane_bytes();
  CK(cudaMemsetAsync(c->scratch, 0, pb * c->nplanes(), c->stream));
  CK(c->L->flux(c->kp, c->A, c->scratch, dir, c->cmax, c->stream));
  CK(cudaMemcpyAsync(F_m, c->scratch, pb * c->kp.nvm, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(F_h, c->scratch + (size_t)c->kp.nvm * c->kp.nc, pb * 5, cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PIP_OK;
}

int pip_source(pip_ctx *c, double dt_coll, double *S_h, double *S_m) {
  if (!c || !S_h || !S_m) return PIP_ERR_NULL;
  if (!c->uploaded || c->mixed || nl_missing(c)) return PIP_ERR_STATE;
  if (set_device(c) || ensure_scratch(c) || ensure_coefficients(c)) return PIP_ERR_CUDA;
  const size_t pb = c->plane_bytes();
  // set_IR type 4: the rates (and ion_pot) of the state as given, as for types 2 and 3
  if (c->kp.irn)
    CK(c->L->nlev_rates(c->kp, c->A, 0, c->kp.ir_type == 0 ? 1 : 0, nullptr, c->ctrl, c->stream));
  CK(c->L->source(c->kp, c->A, c->scratch, dt_coll, c->stream));
  CK(cudaMemcpyAsync(S_m, c->scratch, pb * c->kp.nvm, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(S_h, c->scratch + (size_t)c->kp.nvm * c->kp.nc, pb * 5, cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PIP_OK;
}

int pip_coefficients(pip_ctx *c) {
  if (!c) return PIP_ERR_NULL;
  if (!c->uploaded || nl_missing(c)) return PIP_ERR_STATE;
  if (!c->kp.col_type && !c->kp.irl) return PIP_OK;
  if (set_device(c)) return PIP_ERR_CUDA;
  if (c->kp.irn) {   // set_IR type 4's rates come before the rewrites
    c->coef_valid = false;
    if (ensure_coefficients(c)) return PIP_ERR_CUDA;
    CK(cudaStreamSynchronize(c->stream));
    return PIP_OK;
  }
  CK(c->L->coefficients(c->kp, c->A, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->coef_valid = true;
  return PIP_OK;
}

int pip_get_alpha_c(pip_ctx *c, double *ac) {
  if (!c || !ac) return PIP_ERR_NULL;
  if (!c->uploaded) return PIP_ERR_STATE;
  if (!c->kp.col_type) {
    for (long long q = 0; q < c->kp.nc; ++q) ac[q] = c->p.col;
    return PIP_OK;
  }
  if (set_device(c) || ensure_coefficients(c)) return PIP_ERR_CUDA;
  CK(cudaMemcpyAsync(ac, c->acf, c->plane_bytes(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PIP_OK;
}

int pip_set_alpha_c(pip_ctx *c, const double *ac) {
  if (!c || !ac) return PIP_ERR_NULL;
  if (!c->uploaded) return PIP_ERR_STATE;
  if (!c->kp.col_type) return PIP_OK;
  if (set_device(c)) return PIP_ERR_CUDA;
  CK(cudaMemcpyAsync(c->acf, ac, c->plane_bytes(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->coef_valid = true;
  return PIP_OK;
}

int pip_resi_dt(pip_ctx *c, double *bound) {
  if (!c || !bound) return PIP_ERR_NULL;
  if (!c->kp.resi) return PIP_ERR_PARAM;
  if (c->kp.resi == 1) {
    *bound = c->kp.resi_dt;
    return PIP_OK;
  }
  if (!c->uploaded) return PIP_ERR_STATE;
  if (set_device(c)) return PIP_ERR_CUDA;
  if (ensure_coefficients(c)) return PIP_ERR_CUDA;
  unsigned long long b = 0;
  CK(cudaMemcpyAsync(&b, c->d_resi, sizeof b, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::memcpy(bound, &b, sizeof(double));
  return PIP_OK;
}

int pip_set_resistivity(pip_ctx *c, const double *eta) {
  if (!c || !eta) return PIP_ERR_NULL;
  if (c->kp.resi != 1) return PIP_ERR_PARAM;   // none, or eta computed from the state
  if (set_device(c)) return PIP_ERR_CUDA;
  CK(cudaStreamSynchronize(c->stream));      // no queued kernel still reads the field
  CK(cudaMemcpy(c->etaf, eta, c->plane_bytes(), cudaMemcpyHostToDevice));
  c->kp.resi_dt = resi_bound(c, eta);
  if (c->graph) {                             // the graph holds the old kernel parameters
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
    c->graph_steps = 0;
  }
  return PIP_OK;
}

int pip_fill_ghosts(pip_ctx *c) {
  if (!c) return PIP_ERR_NULL;
  if (!c->uploaded) return PIP_ERR_STATE;
  if (set_device(c)) return PIP_ERR_CUDA;
  CK(to_fp64(c));
  CK(c->L->ghosts(c->kp, c->A, c->stream));
  CK(from_fp64(c));
  CK(cudaStreamSynchronize(c->stream));
  return PIP_OK;
}

int pip_status(pip_ctx *c, int *stop_flag, int *nan_flag) {
  if (!c) return PIP_ERR_NULL;
  if (!c->uploaded) return PIP_ERR_STATE;
  if (set_device(c)) return PIP_ERR_CUDA;
  int h = 0;
  CK(cudaMemsetAsync(c->d_flag, 0, sizeof(int), c->stream));
  CK(to_fp64(c));
  CK(c->L->nan_scan(c->kp, c->A, c->d_flag, c->stream));
  CK(cudaMemcpyAsync(&h, c->d_flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (nan_flag) *nan_flag = h;
  if (stop_flag) *stop_flag = (h || c->last_dt <= 1.0e-12) ? 1 : 0;
  return PIP_OK;
}

int pip_conduction(pip_ctx *c, double dt, int *iters, double *relres) {
  if (!c) return PIP_ERR_NULL;
  if (iters) *iters = 0;
  if (relres) *relres = 0.0;
  if (!c->hc) return PIP_ERR_PARAM;      // context created without flag_heat = 1
  if (!c->uploaded) return PIP_ERR_STATE;
  if (!(dt > 0.0) || !std::isfinite(dt)) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  double *hdt = &c->h_ctrl->dt;
  *hdt = dt;
  CK(cudaMemcpyAsync(c->d_dt, hdt, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  int it = 0, st = 0;
  double rr = 0.0;
  const int r = conduct(c, c->d_dt, &it, &rr, &st);
  if (r != PIP_OK) return r;
  CK(cudaStreamSynchronize(c->stream));
  c->hc_iters = it;
  if (iters) *iters = it;
  if (relres) *relres = rr;
  return st == 0 ? PIP_OK : PIP_ERR_ITER;
}

int pip_set_hc_wait_limit(pip_ctx *c, int polls) {
  if (!c) return PIP_ERR_NULL;
  if (!c->hc) return PIP_ERR_PARAM;
  pip::hc_set_wait_limit(c->hc, polls);
  return PIP_OK;
}

int pip_set_hc_loop(pip_ctx *c, int device_loop) {
  if (!c) return PIP_ERR_NULL;
  if (!c->hc || (device_loop != 0 && device_loop != 1)) return PIP_ERR_PARAM;
  pip::hc_set_loop(c->hc, device_loop);
  return PIP_OK;
}

int pip_set_neighbors(pip_ctx *c, const int neighbor[4]) {
  if (!c || !neighbor) return PIP_ERR_NULL;
  bool any = false;
  for (int f = 0; f < 4; ++f) {
    if (neighbor[f] < -1) return PIP_ERR_PARAM;
    if (f >= 2 * c->kp.ndim && neighbor[f] != -1) return PIP_ERR_PARAM;
    any = any || neighbor[f] >= 0;
  }
  // with eta recomputed at every stage each rank advances its time by its own cfl_resi
  // bound; conduction splits along y only (pip_hcd_*)
  if (any && (c->kp.resi == 2 || c->kp.irn)) return PIP_ERR_PARAM;
  if (c->hc && (neighbor[0] >= 0 || neighbor[1] >= 0)) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  if (c->stream) CK(cudaStreamSynchronize(c->stream));
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
    c->graph_steps = 0;
  }
  build_kparams(c);                  // physical boundaries of every face ...
  for (int f = 0; f < 4; ++f) {      // ... then the exchanged faces get no ghost source
    c->neighbor[f] = neighbor[f];
    if (neighbor[f] < 0) continue;
    int *g = f < 2 ? c->kp.gx[f] : c->kp.gy[f - 2];
    for (int l = 0; l < pip::kMaxMargin; ++l) g[l] = -1;
    (f < 2 ? c->kp.typex[f] : c->kp.typey[f - 2]) = 0;
  }
  c->kp.dx = c->d_dx;
  c->kp.dy = c->d_dy;
  c->kp.rdx = c->d_rdx;
  c->kp.rdy = c->d_rdy;
  c->exchanged = any;
  return PIP_OK;
}

int pip_stage(pip_ctx *c, int stage, double dt, double cmax) {
  if (!c) return PIP_ERR_NULL;
  if (!c->uploaded) return PIP_ERR_STATE;
  if (stage != 1 && stage != 2) return PIP_ERR_PARAM;
  if (!(dt > 0.0) || !std::isfinite(dt) || !std::isfinite(cmax)) return PIP_ERR_PARAM;
  if (stage == 2 && c->last_stage != 1) return PIP_ERR_STATE;
  if (set_device(c)) return PIP_ERR_CUDA;
  if (stage == 1) {
    if (ensure_coefficients(c)) return PIP_ERR_CUDA;
    stage_ctrl_kernel<<<1, 1, 0, c->stream>>>(c->ctrl, dt, cmax);
    CK(cudaGetLastError());
    c->cmax = cmax;
  }
  CK(do_stage(c, stage, 0, 0));
  if (stage == 2 && c->hc && !c->exchanged) {   // with neighbours: pip_hcd_* after the exchange
    CK(cudaMemcpyAsync(c->d_dt, &c->ctrl->dt, sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    int it = 0, st = 0;
    const int r = conduct(c, c->d_dt, &it, nullptr, &st);
    if (r != PIP_OK) return r;
    c->hc_iters = it;
  }
  CK(cudaGetLastError());
  c->last_stage = stage;
  if (stage == 2) c->last_dt = dt;
  return PIP_OK;
}

int pip_set_cmax_scale(pip_ctx *c, double safety_min_d) {
  if (!c) return PIP_ERR_NULL;
  if (!(safety_min_d > 0.0) || !std::isfinite(safety_min_d)) return PIP_ERR_PARAM;
  c->kp.sg_all = safety_min_d;
  if (c->graph) {
    if (set_device(c)) return PIP_ERR_CUDA;
    CK(cudaStreamSynchronize(c->stream));
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
    c->graph_steps = 0;
  }
  return PIP_OK;
}

int pip_dev_begin(pip_ctx *c, int64_t nsteps, double t_end) {
  if (!c) return PIP_ERR_NULL;
  if (!c->uploaded || c->hc) return c->hc ? PIP_ERR_PARAM : PIP_ERR_STATE;
  if (c->kp.irn) return PIP_ERR_PARAM;   // set_IR type 4 steps on the host (pip_run)
  if (nsteps <= 0 && !(t_end > 0.0)) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  CK(cudaStreamSynchronize(c->stream));   // nothing queued still reads the pinned block
  DevCtrl &h = *c->h_ctrl;
  std::memset(&h, 0, sizeof(DevCtrl));
  h.time = c->time;
  h.t_end = t_end > 0.0 ? t_end : 0.0;
  h.nsteps = nsteps > 0 ? nsteps : 0;
  h.cmax = c->cmax;
  reset_slot(h, 0, c->kp);
  reset_slot(h, 1, c->kp);
  if (ensure_coefficients(c)) return PIP_ERR_CUDA;
  if (push_ctrl(c)) return PIP_ERR_CUDA;
  CK(do_cfl(c, 0));                         // the first step's cfl candidates (main.f90:36)
  CK(cudaStreamSynchronize(c->stream));
  c->last_stage = 0;
  c->dev_loop = true;
  return PIP_OK;
}

int pip_dev_stage(pip_ctx *c, int stage) {
  if (!c) return PIP_ERR_NULL;
  if (!c->dev_loop) return PIP_ERR_STATE;
  if (stage != 1 && stage != 2) return PIP_ERR_PARAM;
  if (stage == 2 && c->last_stage != 1) return PIP_ERR_STATE;
  if (set_device(c)) return PIP_ERR_CUDA;
  CK(stage == 1 ? do_stage(c, 1, 1, 0) : do_stage(c, 2, 1, -1));
  c->last_stage = stage;
  return PIP_OK;
}

int pip_dev_stage_split(pip_ctx *c, int stage, void **boundary_stream) {
  if (!c || !boundary_stream) return PIP_ERR_NULL;
  if (!c->dev_loop) return PIP_ERR_STATE;
  if (stage != 1 && stage != 2) return PIP_ERR_PARAM;
  if (c->kp.ndim != 2) return PIP_ERR_PARAM;
  if (stage == 2 && c->last_stage != 1) return PIP_ERR_STATE;
  if (set_device(c)) return PIP_ERR_CUDA;
  if (!c->rows_stream) {
    int lo = 0, hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CK(cudaStreamCreateWithPriority(&c->rows_stream, cudaStreamNonBlocking, hi));
    CK(cudaEventCreateWithFlags(&c->rows_ev[0], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->rows_ev[1], cudaEventDisableTiming));
  }
  // the boundary rows on the high-priority stream, concurrent with the middle rows on the
  // context stream; the context stream then waits for them
  const int epi = stage == 1 ? 0 : -1;
  cudaStream_t s0 = c->stream;
  CK(cudaEventRecord(c->rows_ev[0], s0));
  CK(cudaStreamWaitEvent(c->rows_stream, c->rows_ev[0], 0));
  c->stream = c->rows_stream;
  cudaError_t e = do_stage(c, stage, 1, epi, 1);
  c->stream = s0;
  CK(e);
  CK(cudaEventRecord(c->rows_ev[1], c->rows_stream));
  CK(do_stage(c, stage, 1, epi, 2));
  CK(cudaStreamWaitEvent(s0, c->rows_ev[1], 0));
  c->last_stage = stage;
  *boundary_stream = (void *)c->rows_stream;
  return PIP_OK;
}

int pip_set_halo_stream(pip_ctx *c, void *stream) {
  if (!c) return PIP_ERR_NULL;
  c->halo_stream = static_cast<cudaStream_t>(stream);
  return PIP_OK;
}

int pip_dev_candidates(pip_ctx *c, void **dt_min, void **rho_gr_max) {
  if (!c || !dt_min || !rho_gr_max) return PIP_ERR_NULL;
  *dt_min = (void *)&c->ctrl->red_dt[0];
  *rho_gr_max = (void *)&c->ctrl->red_rho[0];
  return PIP_OK;
}

int pip_dev_poll(pip_ctx *c, int *done, double *time, int64_t *steps) {
  if (!c) return PIP_ERR_NULL;
  if (!c->dev_loop) return PIP_ERR_STATE;
  if (set_device(c)) return PIP_ERR_CUDA;
  if (sync_ctrl_to_host(c)) return PIP_ERR_CUDA;
  const DevCtrl &h = *c->h_ctrl;
  c->time = h.time;
  c->dt = h.dt;
  c->last_dt = h.dt;
  c->cmax = h.cmax;
  if (done) *done = (h.done || h.nan_flag) ? 1 : 0;
  if (time) *time = h.time;
  if (steps) *steps = h.step;
  if (h.nan_flag) return PIP_ERR_NAN;
  if (h.status) return h.status;
  return PIP_OK;
}

int pip_ctx_stream(pip_ctx *c, void **stream) {
  if (!c || !stream) return PIP_ERR_NULL;
  *stream = (void *)c->stream;
  return PIP_OK;
}

namespace {
// The arrays the last stage wrote: stage 1 -> U1 (B, or Bf in the mixed form), otherwise
// the state (A, or the FP32 pair Ahi/Alo).
void halo_arrays(pip_ctx *c, void **a0, void **a1, int *eb) {
  *a1 = nullptr;
  if (c->last_stage == 1) {
    *a0 = c->mixed ? (void *)c->Bf : (void *)c->B;
    *eb = c->mixed ? 4 : 8;
  } else if (c->mixed) {
    *a0 = c->Ahi;
    *a1 = c->Alo;
    *eb = 4;
  } else {
    *a0 = c->A;
    *eb = 8;
  }
}
}  // namespace

int64_t pip_halo_bytes(pip_ctx *c, int face) {
  if (!c || face < 0 || face >= 2 * c->kp.ndim) return 0;
  return (int64_t)pip::halo_elems(c->kp, face) * 8;
}

int pip_halo_pack(pip_ctx *c, int face, void *send, int64_t *bytes) {
  if (!c || !send) return PIP_ERR_NULL;
  if (face < 0 || face >= 2 * c->kp.ndim) return PIP_ERR_PARAM;
  if (!c->uploaded) return PIP_ERR_STATE;
  if (set_device(c)) return PIP_ERR_CUDA;
  void *a0, *a1;
  int eb;
  halo_arrays(c, &a0, &a1, &eb);
  CK(pip::halo_pack(c->kp, face, a0, a1, eb, send, c->halo_stream ? c->halo_stream : c->stream));
  if (bytes) *bytes = (int64_t)pip::halo_elems(c->kp, face) * eb * (a1 ? 2 : 1);
  return PIP_OK;
}

int pip_halo_unpack(pip_ctx *c, int face, const void *recv, int64_t bytes) {
  if (!c || !recv) return PIP_ERR_NULL;
  if (face < 0 || face >= 2 * c->kp.ndim) return PIP_ERR_PARAM;
  if (!c->uploaded) return PIP_ERR_STATE;
  void *a0, *a1;
  int eb;
  halo_arrays(c, &a0, &a1, &eb);
  if (bytes != (int64_t)pip::halo_elems(c->kp, face) * eb * (a1 ? 2 : 1)) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  CK(pip::halo_unpack(c->kp, face, a0, a1, eb, recv,
                      c->halo_stream ? c->halo_stream : c->stream));
  return PIP_OK;
}

int pip_set_nlevel(pip_ctx *c, const pip_nlevel *cfg, const double *table, int64_t nrows) {
  if (!c || !cfg || !table) return PIP_ERR_NULL;
  if (!c->kp.irn) return PIP_ERR_PARAM;
  if (cfg->n_levels != 5 || cfg->flag_rad < 0 || cfg->flag_rad > 1) return PIP_ERR_PARAM;
  if (cfg->deriv != 0 && cfg->deriv != 1 && cfg->deriv != 4) return PIP_ERR_PARAM;
  if (nrows < 3 || !(cfg->n0fac != 0.0) || !(cfg->f_p_ini != 0.0) || !std::isfinite(cfg->f_p_p_ini))
    return PIP_ERR_PARAM;
  for (int64_t r = 0; r + 1 < nrows; ++r)
    if (!(table[4 * (r + 1)] > table[4 * r])) return PIP_ERR_PARAM;   // abscissae increase
  if (set_device(c)) return PIP_ERR_CUDA;
  CK(cudaStreamSynchronize(c->stream));
  cudaFree(c->nl_tab);
  cudaFree(c->nl_rtab);
  c->nl_tab = nullptr;
  c->nl_rtab = nullptr;
  CK(cudaMalloc(&c->nl_tab, sizeof(double) * 4 * (size_t)nrows));
  CK(cudaMemcpy(c->nl_tab, table, sizeof(double) * 4 * (size_t)nrows, cudaMemcpyHostToDevice));
  {
    // quadratic-interpolation denominators of each row's three-row stencil (FMA build)
    std::vector<double> rt(4 * (size_t)nrows, 0.0);
    for (int64_t r = 0; r + 2 < nrows; ++r) {
      const double x0 = table[4 * r], x1 = table[4 * (r + 1)], x2 = table[4 * (r + 2)];
      rt[4 * r] = 1.0 / ((x0 - x1) * (x0 - x2));
      rt[4 * r + 1] = 1.0 / ((x1 - x0) * (x1 - x2));
      rt[4 * r + 2] = 1.0 / ((x2 - x0) * (x2 - x1));
    }
    CK(cudaMalloc(&c->nl_rtab, sizeof(double) * rt.size()));
    CK(cudaMemcpy(c->nl_rtab, rt.data(), sizeof(double) * rt.size(), cudaMemcpyHostToDevice));
  }
  pip::NlevConst k;
  pip::nlev_constants(&k);
  CK(cudaMemcpy(c->nl_k, &k, sizeof k, cudaMemcpyHostToDevice));
  KParams &kp = c->kp;
  kp.nl_tab = c->nl_tab;
  kp.nl_ntab = nrows;
  kp.nl_xmin = table[0];
  kp.nl_xrange = table[4 * (nrows - 1)] - table[0];
  kp.nl_rtab = c->nl_rtab;
  kp.nl_xsc = (double)nrows / kp.nl_xrange;
  kp.nl_deriv = cfg->deriv;
  kp.nl_n0fac = cfg->n0fac;
  // tfac of set_IR type 4 (PIP_rot.f90:240-248); 5.0/3.0 is a default-real quotient there
  kp.nl_tfac = c->p.flag_col % 2 == 1
                   ? c->p.t_norm / ((double)(5.0f / 3.0f) * cfg->f_p_p_ini / cfg->f_p_ini)
                   : c->p.beta / 2.0 * cfg->f_p_p_ini * 5.0 / 6.0 / cfg->f_p_ini;
  c->nl_ready = true;
  c->nl_init = false;
  c->coef_valid = false;
  return PIP_OK;
}

int pip_set_nexcite(pip_ctx *c, const double *nexcite) {
  if (!c || !nexcite) return PIP_ERR_NULL;
  if (!c->kp.irn) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  CK(cudaMemcpyAsync(c->kp.nl_nex, nexcite, 6 * c->plane_bytes(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PIP_OK;
}

int pip_get_nexcite(pip_ctx *c, double *nexcite) {
  if (!c || !nexcite) return PIP_ERR_NULL;
  if (!c->kp.irn) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  CK(cudaMemcpyAsync(nexcite, c->kp.nl_nex, 6 * c->plane_bytes(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PIP_OK;
}

int pip_get_colrat(pip_ctx *c, double *colrat) {
  if (!c || !colrat) return PIP_ERR_NULL;
  if (!c->kp.irn) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  CK(cudaMemcpyAsync(colrat, c->nl_cr, 36 * c->plane_bytes(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PIP_OK;
}

int pip_get_ion_pot(pip_ctx *c, double *ion_pot) {
  if (!c || !ion_pot) return PIP_ERR_NULL;
  if (!c->kp.irn) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  CK(cudaMemcpyAsync(ion_pot, c->nl_ip, c->plane_bytes(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PIP_OK;
}

int pip_get_ir_rates(pip_ctx *c, double *gm_ion, double *gm_rec) {
  if (!c || !gm_ion || !gm_rec) return PIP_ERR_NULL;
  if (!c->irg) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  CK(cudaMemcpyAsync(gm_ion, c->irg, c->plane_bytes(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(gm_rec, c->irg + c->kp.nc, c->plane_bytes(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PIP_OK;
}

int pip_nlevel_gm_rec_ref(pip_ctx *c, double *gm_rec_ref) {
  if (!c || !gm_rec_ref) return PIP_ERR_NULL;
  if (!c->kp.irn) return PIP_ERR_PARAM;
  if (!c->nl_init) return PIP_ERR_STATE;
  *gm_rec_ref = c->kp.nl_gref;
  return PIP_OK;
}

__global__ void set_double_kernel(double *dst, double v) { *dst = v; }

int pip_hcd_begin(pip_ctx *c, double dt, double sums[2]) {
  if (!c || !sums) return PIP_ERR_NULL;
  if (!c->hc) return PIP_ERR_PARAM;
  if (!c->uploaded) return PIP_ERR_STATE;
  if (!(dt > 0.0) || !std::isfinite(dt)) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  CK(to_fp64(c));
  set_double_kernel<<<1, 1, 0, c->stream>>>(c->d_dt, dt);
  CK(cudaGetLastError());
  CK(pip::hcd_begin(c->hc, c->kp, c->A, c->d_dt, c->stream, sums));
  return PIP_OK;
}

int pip_hcd_phase(pip_ctx *c, int phase, const double coef[2], double sums[2]) {
  if (!c) return PIP_ERR_NULL;
  if (!c->hc) return PIP_ERR_PARAM;
  if (phase < 0 || phase > 5) return PIP_ERR_PARAM;
  if ((phase == 1 || phase == 2 || phase == 4) && !sums) return PIP_ERR_NULL;
  if ((phase == 2 || phase == 3 || phase == 5) && !coef) return PIP_ERR_NULL;
  if (set_device(c)) return PIP_ERR_CUDA;
  double dummy[2];
  CK(pip::hcd_phase(c->hc, c->kp, phase, coef, c->stream, sums ? sums : dummy));
  return PIP_OK;
}

int64_t pip_hcd_row_bytes(pip_ctx *c) { return c ? (int64_t)sizeof(double) * c->kp.ix : 0; }

int pip_hcd_pack(pip_ctx *c, int vec, int face, void *send) {
  if (!c || !send) return PIP_ERR_NULL;
  if (!c->hc || (face != 2 && face != 3) || vec < 0 || vec > 2) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  const int row = face == 2 ? c->kp.m1 : c->kp.m1 + c->kp.ny - 1;   // the neighbour's halo row
  const double *v = pip::hcd_vector(c->hc, vec) + (size_t)row * c->kp.ix;
  CK(cudaMemcpyAsync(send, v, sizeof(double) * c->kp.ix, cudaMemcpyDeviceToDevice, c->stream));
  return PIP_OK;
}

int pip_hcd_unpack(pip_ctx *c, int vec, int face, const void *recv) {
  if (!c || !recv) return PIP_ERR_NULL;
  if (!c->hc || (face != 2 && face != 3) || vec < 0 || vec > 2) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  const int row = face == 2 ? c->kp.m1 - 1 : c->kp.m1 + c->kp.ny;
  double *v = pip::hcd_vector(c->hc, vec) + (size_t)row * c->kp.ix;
  CK(cudaMemcpyAsync(v, recv, sizeof(double) * c->kp.ix, cudaMemcpyDeviceToDevice, c->stream));
  return PIP_OK;
}

int pip_hcd_end(pip_ctx *c, int iters) {
  if (!c) return PIP_ERR_NULL;
  if (!c->hc) return PIP_ERR_PARAM;
  if (set_device(c)) return PIP_ERR_CUDA;
  CK(pip::hcd_end(c->hc, c->kp, c->A, c->stream));
  CK(c->L->ghosts(c->kp, c->A, c->stream));   // physical faces; the caller exchanges the rest
  CK(from_fp64(c));
  CK(cudaStreamSynchronize(c->stream));
  c->hc_iters = iters;
  return PIP_OK;
}

int pip_last_cuda_error(void) { return g_last_cuda_error; }

const char *pip_strerror(int code) {
  switch (code) {
    case PIP_OK: return "ok";
    case PIP_ERR_PARAM: return "unsupported or inconsistent parameters";
    case PIP_ERR_CUDA: return "CUDA runtime error";
    case PIP_ERR_NAN: return "NaN in the state";
    case PIP_ERR_DT: return "time step <= 1e-12";
    case PIP_ERR_ITER: return "iteration limit reached";
    case PIP_ERR_STATE: return "call out of order";
    case PIP_ERR_NOMEM: return "device allocation failed";
    case PIP_ERR_NULL: return "NULL argument";
    case PIP_ERR_RATE: return "negative rate of the 6-level hydrogen model";
    default: return "unknown status";
  }
}

}  // extern "C"
