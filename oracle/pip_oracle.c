/*
 * pip_oracle.c -- TEST INFRASTRUCTURE ONLY (see pip_oracle.h).
 *
 * FP64 CPU restatement of the PIP two-fluid step.  Each routine names the Fortran it
 * restates.  Arrays use the Fortran layout U(ix,jx,kx,nvar), column-major, 0-based here:
 * element (i,j,k,n) sits at i + ix*(j + jx*(k + kx*n)).  Whole-array passes with
 * temporaries, as the Fortran does; expressions keep the Fortran evaluation order
 * (left-to-right, parentheses as written) and the file is compiled without FMA
 * contraction, so results match an -O2 x86-64 gfortran build up to libm differences.
 */
#include "pip_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TINY 1.0e-20                 /* Globalvar.f90:101 */
#define HLLC_EPSI 1.0e-10            /* HLL_rot.f90:12 */
#define HLLC_ACC 1.03                /* HLL_rot.f90:12 */
#define HLLG_FACTOR 1.001            /* HLL_rot.f90:702 */
#define MU_P 0.5                     /* initialize_collisional, PIP_rot.f90:35 */
#define MU_N 1.0                     /* PIP_rot.f90:36 */
#define PI_REF 3.1415926535897932    /* Parameters.f90:2 */

struct orc_ctx {
  pip_params p;
  int ix, jx, kx, nh, nm;
  size_t nc;                         /* cells */
  double *dx, *dy, *dz;
  double *U_h, *U_m;
  double *gm_ion, *gm_rec;           /* IR rates (PIP_IR_POWERLAW) */
  int sym_m[6][9], sym_h[6][5];      /* set_sym_mhd / set_sym_hd */
  double cmax, time, last_dt;
  int neighbor[6];                   /* set_mpi_neighbor: rank across each face, -1 physical */
  double *U_h0, *U_m0;               /* run_solver's U0 between orc_stage calls */
  double stage_dt;
  int col_type;                      /* initialize_collisional: flag_col 2..7 -> 1..6 */
  double *ac;                        /* alpha_c per cell (globalvar ac) for col_type >= 1 */
  int init_done;                     /* set_coefficients(U_h,U_m,0) has run */
  int resi;                          /* flag_resi 1: resistive flux with a fixed eta field;
                                        2: eta from set_resistivity at every RK stage */
  double *eta;                       /* globalvar eta (set_resistivity), nc values */
  /* set_IR type 4, the 6-level hydrogen model */
  int nlev_deriv;                    /* convective derivative: 0 none, 1 two-point, 4 five-point */
  double n0fac, f_p_ini, f_p_p_ini;  /* globalvar normalisation of the model */
  double *etab;                      /* expinttab (4 x netab, column-major) */
  long netab;
  double *nex;                       /* Nexcite (ix,jx,kx,6) */
  double *colrat;                    /* colrat (ix,jx,kx,6,6) */
  double *ion_pot;                   /* globalvar ion_pot: the last irgetionpot, nc values */
  double gm_rec_ref;                 /* Gm_rec_ref */
  int nlev_init;                     /* the prologue's block of set_IR type 4 has run */
  /* conduction of a decomposed run (orc_hcd_*): te, b, r, r0, p, Ap, t, the matrix and the
   * primitives of the write-back */
  double *hcd;                       /* 7 vectors then 9 matrix planes then 8 primitives */
  int nlev_bad;                      /* a negative rate (the reference stops there) */
  struct {
    double gw[6], eion[6], rn[6], bn[6];
    double xrat[5][5], enn[5][5], rnn[5][5], ann[5][5], bnn[5][5], lgt[5][5];
    double an0[5], bn0[5], lgi[5];
  } nk;                              /* get_col_ion_coeff's cell-independent coefficients */
};

static void ensure_coefficients(orc_ctx *c);
static double cfl_resi(orc_ctx *c, double dt);

static int g_threads = 1;

void orc_set_threads(int n) {
  g_threads = n > 0 ? n : 1;
#ifdef _OPENMP
  omp_set_num_threads(g_threads);
#endif
}
int orc_get_threads(void) { return g_threads; }

static inline double fmx(double a, double b) { return a > b ? a : b; }
static inline double fmn(double a, double b) { return a < b ? a : b; }
static inline double sgn1(double b) { return copysign(1.0, b); }  /* sign(1.0d0,b) */

#define AT(c, i, j, k) ((size_t)(i) + (size_t)(c)->ix * ((size_t)(j) + (size_t)(c)->jx * (size_t)(k)))

/* ---------------------------------------------------------------- boundary tables */

/* set_sym_mhd, Boundary_rot.f90:239-294 (dir is 1-based, face index f 0-based). */
static void set_sym_mhd(orc_ctx *c) {
  const pip_params *p = &c->p;
  for (int f = 0; f < 6; ++f)
    for (int n = 0; n < 9; ++n) c->sym_m[f][n] = 1;
  for (int f = 0; f < 2 * p->ndim; ++f) {
    int dir = f / 2 + 1, b = p->flag_bnd[f];
    /* Fortran indices below are 1-based variable numbers; subtract 1. */
    if (b == 2) {
      c->sym_m[f][1 + dir - 1] = -1;
      c->sym_m[f][5 + dir - 1] = -1;
    } else if (b == 3) {
      c->sym_m[f][1 + dir - 1] = -1;
      c->sym_m[f][6 + dir % 3 - 1] = -1;
      c->sym_m[f][2 + (dir + 1) % 3 - 1] = -1;
    } else if (b == 4) {
      c->sym_m[f][1 + dir - 1] = -1;
      c->sym_m[f][6 + (dir + 1) % 3 - 1] = -1;
      c->sym_m[f][2 + dir % 3 - 1] = -1;
    } else if (b == 5) {
      c->sym_m[f][1 + dir - 1] = -1;
      c->sym_m[f][5 + dir - 1] = -1;
      c->sym_m[f][2 + (dir + 1) % 3 - 1] = -1;
      c->sym_m[f][6 + (dir + 1) % 3 - 1] = -1;
    } else if (b == 6) {
      c->sym_m[f][1 + dir - 1] = -1;
      c->sym_m[f][6 + dir % 3 - 1] = -1;
      c->sym_m[f][6 + (dir + 1) % 3 - 1] = -1;
    } else if (b == 7) {
      c->sym_m[f][1] = -1;
      c->sym_m[f][2] = -1;
      c->sym_m[f][3] = -1;
    }
  }
  if (p->flag_divb == 1) {
    for (int f = 0; f < 2 * p->ndim; ++f) {
      int b = p->flag_bnd[f];
      if (b == 2 || b == 20 || b == 5) c->sym_m[f][8] = 1;
      else if (b == 3 || b == 4 || b == 6 || b == 7) c->sym_m[f][8] = -1;
    }
  }
}

/* set_sym_hd, Boundary_rot.f90:296-320. */
static void set_sym_hd(orc_ctx *c) {
  const pip_params *p = &c->p;
  for (int f = 0; f < 6; ++f)
    for (int n = 0; n < 5; ++n) c->sym_h[f][n] = 1;
  for (int f = 0; f < 2 * p->ndim; ++f) {
    int dir = f / 2 + 1, b = p->flag_bnd[f];
    if (b == 2 || b == 20) {
      c->sym_h[f][1 + dir - 1] = -1;
    } else if (b == 3) {
      c->sym_h[f][1 + dir - 1] = -1;
      c->sym_h[f][2 + (dir + 1) % 3 - 1] = -1;
    } else if (b == 4) {
      c->sym_h[f][1 + dir - 1] = -1;
      c->sym_h[f][2 + dir % 3 - 1] = -1;
    } else if (b == 5) {
      c->sym_h[f][1 + dir - 1] = -1;
      c->sym_h[f][2 + (dir + 1) % 3 - 1] = -1;
    } else if (b == 6) {
      c->sym_h[f][1 + dir - 1] = -1;
    }
  }
}

/* boundary_control, Boundary_rot.f90:323-402, for one face and one species. */
static void boundary_control(orc_ctx *c, double *U, int nvar, int dir, int upper, const int *sym,
                             int type) {
  int ig[3] = {c->ix, c->jx, c->kx};
  int sl[3], el[3], dl[3], sr[3], er[3], dr[3];
  const int *margin = c->p.margin;
  for (int a = 0; a < 3; ++a) {
    if (dir == a + 1) {
      if (!upper) {
        sl[a] = 1; el[a] = margin[a]; dl[a] = 1;
        if (type == 1) { sr[a] = ig[a] - 2 * margin[a] + 1; er[a] = ig[a] - margin[a]; dr[a] = 1; }
        else if (type == 2) { sr[a] = 2 * margin[a]; er[a] = margin[a] + 1; dr[a] = -1; }
        else { sr[a] = margin[a] + 1; er[a] = margin[a] + 1; dr[a] = 1; }
      } else {
        sl[a] = ig[a] - margin[a] + 1; el[a] = ig[a]; dl[a] = 1;
        if (type == 1) { sr[a] = margin[a] + 1; er[a] = 2 * margin[a]; dr[a] = 1; }
        else if (type == 2) { sr[a] = ig[a] - margin[a]; er[a] = ig[a] - margin[a] * 2 + 1; dr[a] = -1; }
        else { sr[a] = ig[a] - margin[a]; er[a] = ig[a] - margin[a]; dr[a] = 1; }
      }
    } else {
      sl[a] = 1; el[a] = ig[a]; dl[a] = 1;
      sr[a] = 1; er[a] = ig[a]; dr[a] = 1;
    }
  }
  int same = 1;
  for (int a = 0; a < 3; ++a)
    if (el[a] - sl[a] != abs(er[a] - sr[a])) same = 0;
  size_t nc = c->nc;
  if (same) {
    for (int n = 0; n < nvar; ++n) {
      double s = (double)sym[n];
      for (int k = 0; k <= el[2] - sl[2]; ++k)
        for (int j = 0; j <= el[1] - sl[1]; ++j)
          for (int i = 0; i <= el[0] - sl[0]; ++i) {
            int li = sl[0] + i * dl[0] - 1, lj = sl[1] + j * dl[1] - 1, lk = sl[2] + k * dl[2] - 1;
            int ri = sr[0] + i * dr[0] - 1, rj = sr[1] + j * dr[1] - 1, rk = sr[2] + k * dr[2] - 1;
            U[AT(c, li, lj, lk) + n * nc] = s * U[AT(c, ri, rj, rk) + n * nc];
          }
    }
  } else if (type == 10) {
    /* free boundary: every ghost layer copies the first interior layer (no sign flip) */
    int m = margin[dir - 1], src = sr[dir - 1] - 1;
    for (int n = 0; n < nvar; ++n)
      for (int q = 0; q < m; ++q) {
        int dst = sl[dir - 1] - 1 + q;
        if (dir == 1) {
          for (int k = 0; k < c->kx; ++k)
            for (int j = 0; j < c->jx; ++j)
              U[AT(c, dst, j, k) + n * nc] = U[AT(c, src, j, k) + n * nc];
        } else if (dir == 2) {
          for (int k = 0; k < c->kx; ++k)
            for (int i = 0; i < c->ix; ++i)
              U[AT(c, i, dst, k) + n * nc] = U[AT(c, i, src, k) + n * nc];
        } else {
          for (int j = 0; j < c->jx; ++j)
            for (int i = 0; i < c->ix; ++i)
              U[AT(c, i, j, dst) + n * nc] = U[AT(c, i, j, src) + n * nc];
        }
      }
  }
}

/* Type mapping of MHDbnd/HDbnd, Boundary_rot.f90:54-125. */
static int bnd_type(int code) {
  if (code == 3 || code == 4 || code == 5 || code == 6 || code == 7 || code == 11) return 2;
  return code;
}

/* PIPbnd, Boundary_rot.f90:34-52, without its mpi_bnd: MHDbnd/HDbnd on the faces whose
 * neighbor is -1 (:80-90); the faces with a neighbouring rank are left to the caller's
 * halo exchange. */
void orc_bnd(orc_ctx *c) {
  for (int f = 0; f < 2 * c->p.ndim; ++f)
    if (c->neighbor[f] == -1)
      boundary_control(c, c->U_m, c->nm, f / 2 + 1, f % 2, c->sym_m[f], bnd_type(c->p.flag_bnd[f]));
  for (int f = 0; f < 2 * c->p.ndim; ++f)
    if (c->neighbor[f] == -1)
      boundary_control(c, c->U_h, c->nh, f / 2 + 1, f % 2, c->sym_h[f], bnd_type(c->p.flag_bnd[f]));
}

/* set_mpi_neighbor (MPI_rot.f90:90-126) for faces x-, x+, y-, y+. */
void orc_set_neighbors(orc_ctx *c, const int nb[4]) {
  for (int f = 0; f < 4; ++f) c->neighbor[f] = nb[f];
}

/* ---------------------------------------------------------------- conversions */

/* u2v_hd, HLL_rot.f90:1136-1156. */
static void u2v_hd(const orc_ctx *c, const double *U, double *V) {
  const double gm = c->p.gm, ro_lim = c->p.ro_lim, pr_lim = c->p.pr_lim;
  size_t nc = c->nc;
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < nc; ++q) {
    double ro = fmx(U[q], ro_lim);
    double roi = 1.0 / ro;
    double m1 = U[q + nc], m2 = U[q + 2 * nc], m3 = U[q + 3 * nc];
    V[q] = ro;
    V[q + nc] = m1 * roi;
    V[q + 2 * nc] = m2 * roi;
    V[q + 3 * nc] = m3 * roi;
    double pr = (gm - 1.0) * (U[q + 4 * nc] - 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) * roi);
    if (pr < pr_lim) pr = pr_lim;
    V[q + 4 * nc] = pr;
  }
}

/* u2v_mhd, HLL_rot.f90:1159-1186. */
static void u2v_mhd(const orc_ctx *c, const double *U, double *V) {
  const double gm = c->p.gm, ro_lim = c->p.ro_lim, pr_lim = c->p.pr_lim;
  size_t nc = c->nc;
  int divb = c->p.flag_divb == 1;
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < nc; ++q) {
    double ro = fmx(U[q], ro_lim);
    double roi = 1.0 / ro;
    double m1 = U[q + nc], m2 = U[q + 2 * nc], m3 = U[q + 3 * nc];
    double b1 = U[q + 5 * nc], b2 = U[q + 6 * nc], b3 = U[q + 7 * nc];
    V[q] = ro;
    V[q + nc] = m1 * roi;
    V[q + 2 * nc] = m2 * roi;
    V[q + 3 * nc] = m3 * roi;
    double pr = (gm - 1.0) * (U[q + 4 * nc] - 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) * roi -
                              0.5 * (b1 * b1 + b2 * b2 + b3 * b3));
    if (pr < pr_lim) pr = pr_lim;
    V[q + 4 * nc] = pr;
    V[q + 5 * nc] = b1;
    V[q + 6 * nc] = b2;
    V[q + 7 * nc] = b3;
    if (divb) V[q + 8 * nc] = U[q + 8 * nc];
  }
}

/* v2u_1, HLL_rot.f90:1189-1215. */
static void v2u_1(const double *v, double *u, int mhd, int divb, double gm) {
  u[0] = v[0];
  u[1] = v[0] * v[1];
  u[2] = v[0] * v[2];
  u[3] = v[0] * v[3];
  if (!mhd) {
    u[4] = v[4] / (gm - 1.0) + 0.5 * v[0] * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]);
  } else {
    u[5] = v[5];
    u[6] = v[6];
    u[7] = v[7];
    u[4] = v[4] / (gm - 1.0) + 0.5 * v[0] * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]) +
           0.5 * (v[5] * v[5] + v[6] * v[6] + v[7] * v[7]);
    if (divb) u[8] = v[8];
  }
}

/* cq2pv_hd, Scheme_rot.f90:132-150 (rewrites U; returns the primitive arrays). */
static void cq2pv_hd(const orc_ctx *c, double *U, double *de, double *vx, double *vy, double *vz,
                     double *pr) {
  const double gm = c->p.gm, ro_lim = c->p.ro_lim, pr_lim = c->p.pr_lim;
  size_t nc = c->nc;
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < nc; ++q) {
    double d = U[q];
    double ux = U[q + nc] / d, uy = U[q + 2 * nc] / d, uz = U[q + 3 * nc] / d;
    double p = (gm - 1.0) * (U[q + 4 * nc] - 0.5 * d * (ux * ux + uy * uy + uz * uz));
    p = fmx(p, pr_lim);
    d = fmx(d, ro_lim);
    U[q] = d;
    U[q + nc] = ux * d;
    U[q + 2 * nc] = uy * d;
    U[q + 3 * nc] = uz * d;
    U[q + 4 * nc] = p / (gm - 1.0) + 0.5 * d * (ux * ux + uy * uy + uz * uz);
    de[q] = d; vx[q] = ux; vy[q] = uy; vz[q] = uz; pr[q] = p;
  }
}

/* cq2pv_mhd, Scheme_rot.f90:153-179. */
static void cq2pv_mhd(const orc_ctx *c, double *U, double *de, double *vx, double *vy, double *vz,
                      double *pr, double *bx, double *by, double *bz) {
  const double gm = c->p.gm, ro_lim = c->p.ro_lim, pr_lim = c->p.pr_lim;
  size_t nc = c->nc;
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < nc; ++q) {
    double d = U[q];
    double ux = U[q + nc] / d, uy = U[q + 2 * nc] / d, uz = U[q + 3 * nc] / d;
    double b1 = U[q + 5 * nc], b2 = U[q + 6 * nc], b3 = U[q + 7 * nc];
    double p = (gm - 1.0) * (U[q + 4 * nc] - 0.5 * d * (ux * ux + uy * uy + uz * uz) -
                             0.5 * (b1 * b1 + b2 * b2 + b3 * b3));
    p = fmx(p, pr_lim);
    d = fmx(d, ro_lim);
    U[q] = d;
    U[q + nc] = ux * d;
    U[q + 2 * nc] = uy * d;
    U[q + 3 * nc] = uz * d;
    U[q + 4 * nc] = p / (gm - 1.0) + 0.5 * d * (ux * ux + uy * uy + uz * uz) +
                    0.5 * (b1 * b1 + b2 * b2 + b3 * b3);
    de[q] = d; vx[q] = ux; vy[q] = uy; vz[q] = uz; pr[q] = p;
    if (bx) { bx[q] = b1; by[q] = b2; bz[q] = b3; }
  }
}

/* ---------------------------------------------------------------- reconstruction */

/* get_Side (HLL_rot.f90:15-63) with minmod_func (Util_rot.f90:59-76), s_order=2. */
static void get_side(const orc_ctx *c, const double *V, double *VL, double *VR, int dir, int nvar) {
  int ix = c->ix, jx = c->jx, kx = c->kx;
  size_t nc = c->nc;
  memset(VL, 0, sizeof(double) * nc * nvar);
  memset(VR, 0, sizeof(double) * nc * nvar);
  int len = dir == 1 ? ix : (dir == 2 ? jx : kx);
  size_t stride = dir == 1 ? 1 : (dir == 2 ? (size_t)ix : (size_t)ix * jx);
#pragma omp parallel for schedule(static)
  for (int n = 0; n < nvar; ++n) {
    for (int k = 0; k < (dir == 3 ? 1 : kx); ++k)
      for (int j = 0; j < (dir == 2 ? 1 : jx); ++j)
        for (int i = 0; i < (dir == 1 ? 1 : ix); ++i) {
          size_t base = AT(c, i, j, k) + n * nc;
          for (int s = 1; s <= len - 2; ++s) {
            double v0 = V[base + (s - 1) * stride], v1 = V[base + s * stride],
                   v2 = V[base + (s + 1) * stride];
            double X = v2 - v1, Y = v1 - v0;
            double SX = sgn1(X);
            double du = SX * fmx(0.0, fmn(fabs(X), SX * Y));
            VL[base + s * stride] = v1 + 0.5 * du;
            VR[base + (s - 1) * stride] = v1 - 0.5 * du;
          }
        }
  }
  for (size_t q = 0; q < nc; ++q) {
    VL[q] = fmx(VL[q], c->p.ro_lim);
    VR[q] = fmx(VR[q], c->p.ro_lim);
  }
}

/* ---------------------------------------------------------------- Riemann solvers */

/* hllc_flux, HLL_rot.f90:615-687. */
static void hllc_flux(const double *v_l, const double *v_r, double *flx, double gm) {
  double u_l[5], u_r[5], flx_l[5], flx_r[5], st_l[5], st_r[5];
  v2u_1(v_l, u_l, 0, 0, gm);
  v2u_1(v_r, u_r, 0, 0, gm);
  double pr_l = v_l[4], pr_r = v_r[4];
  flx_l[0] = u_l[1];
  flx_r[0] = u_r[1];
  flx_l[1] = pr_l + u_l[1] * u_l[1] / u_l[0];
  flx_r[1] = pr_r + u_r[1] * u_r[1] / u_r[0];
  flx_l[2] = u_l[1] * u_l[2] / u_l[0];
  flx_r[2] = u_r[1] * u_r[2] / u_r[0];
  flx_l[3] = u_l[1] * u_l[3] / u_l[0];
  flx_r[3] = u_r[1] * u_r[3] / u_r[0];
  flx_l[4] = u_l[1] * (u_l[4] + pr_l) / u_l[0];
  flx_r[4] = u_r[1] * (u_r[4] + pr_r) / u_r[0];
  double cs_l = sqrt(gm * pr_l / u_l[0]);
  double cs_r = sqrt(gm * pr_r / u_r[0]);
  double vn_l = u_l[1] / u_l[0];
  double vn_r = u_r[1] / u_r[0];
  double sl = HLLC_ACC * fmn(vn_l - cs_l, vn_r - cs_r);
  double sr = HLLC_ACC * fmx(vn_l + cs_l, vn_r + cs_r);
  double sm = (u_r[1] * (sr - vn_r) - u_l[1] * (sl - vn_l) + pr_l - pr_r) /
              (u_r[0] * (sr - vn_r) - u_l[0] * (sl - vn_l));
  double pr_m = sm * u_l[0] * (sl - vn_l) - u_l[1] * (sl - vn_l) + pr_l;
  st_l[0] = u_l[0] * (sl - vn_l) / (sl - sm);
  st_r[0] = u_r[0] * (sr - vn_r) / (sr - sm);
  st_l[1] = st_l[0] * sm;
  st_r[1] = st_r[0] * sm;
  st_l[2] = st_l[0] * u_l[2] / u_l[0];
  st_r[2] = st_r[0] * u_r[2] / u_r[0];
  st_l[3] = st_l[0] * u_l[3] / u_l[0];
  st_r[3] = st_r[0] * u_r[3] / u_r[0];
  st_l[4] = ((sl - vn_l) * u_l[4] - pr_l * vn_l + pr_m * sm) / (sl - sm);
  st_r[4] = ((sr - vn_r) * u_r[4] - pr_r * vn_r + pr_m * sm) / (sr - sm);
  double thl = (fabs(sl) + sl) / fmx(2.0 * sl, HLLC_EPSI);
  double thm = (fabs(sm) + sm) / fmx(2.0 * sm, HLLC_EPSI);
  double thr = 1.0 - (fabs(sr) + sr) / fmx(2.0 * sr, HLLC_EPSI);
  for (int n = 0; n < 5; ++n)
    flx[n] = thr * flx_r[n] + thl * flx_l[n] +
             (1.0 - thl - thr) * (thm * (flx_l[n] + sl * (st_l[n] - u_l[n])) +
                                  (1.0 - thm) * (flx_r[n] + sr * (st_r[n] - u_r[n])));
}

/* hlld_flux, HLL_rot.f90:691-910 (Miyoshi-Kusano HLLD with HLLC-G fallback). */
static void hlld_flux(const double *v_l, const double *v_r, double *flx, int nvar, double gm,
                      int divb, double cmax) {
  double u_l[9], u_r[9], flx_l[9], flx_r[9], u_hll[9], u_l1[9], u_r1[9], u2[9];
  for (int n = 0; n < 9; ++n) { flx[n] = 0.0; flx_l[n] = 0.0; flx_r[n] = 0.0; }
  (void)nvar;
  v2u_1(v_l, u_l, 1, divb, gm);
  v2u_1(v_r, u_r, 1, divb, gm);

  double b2_l = (v_l[5] * v_l[5] + v_l[6] * v_l[6] + v_l[7] * v_l[7]);
  double pt_l = v_l[4] + 0.5 * b2_l;
  double vbL = v_l[1] * v_l[5] + v_l[2] * v_l[6] + v_l[3] * v_l[7];
  flx_l[0] = v_l[0] * v_l[1];
  flx_l[1] = v_l[0] * (v_l[1] * v_l[1]) + v_l[4] + 0.5 * b2_l - v_l[5] * v_l[5];
  flx_l[2] = v_l[0] * v_l[1] * v_l[2] - v_l[5] * v_l[6];
  flx_l[3] = v_l[0] * v_l[1] * v_l[3] - v_l[5] * v_l[7];
  flx_l[4] = (u_l[4] + pt_l) * v_l[1] - vbL * v_l[5];
  flx_l[5] = 0.0;
  flx_l[6] = v_l[1] * v_l[6] - v_l[5] * v_l[2];
  flx_l[7] = v_l[1] * v_l[7] - v_l[5] * v_l[3];

  double b2_r = (v_r[5] * v_r[5] + v_r[6] * v_r[6] + v_r[7] * v_r[7]);
  double pt_r = v_r[4] + 0.5 * b2_r;
  double vbR = v_r[1] * v_r[5] + v_r[2] * v_r[6] + v_r[3] * v_r[7];
  flx_r[0] = v_r[0] * v_r[1];
  flx_r[1] = v_r[0] * (v_r[1] * v_r[1]) + v_r[4] + 0.5 * b2_r - v_r[5] * v_r[5];
  flx_r[2] = v_r[0] * v_r[1] * v_r[2] - v_r[5] * v_r[6];
  flx_r[3] = v_r[0] * v_r[1] * v_r[3] - v_r[5] * v_r[7];
  flx_r[4] = (u_r[4] + pt_r) * v_r[1] - vbR * v_r[5];
  flx_r[5] = 0.0;
  flx_r[6] = v_r[1] * v_r[6] - v_r[5] * v_r[2];
  flx_r[7] = v_r[1] * v_r[7] - v_r[5] * v_r[3];

  /* fast mode wave speed */
  double f1 = gm * v_l[4];
  double f2 = 4.0 * f1 * (v_l[5] * v_l[5]);
  double vf_l = sqrt(((f1 + b2_l) + sqrt(fmx((f1 + b2_l) * (f1 + b2_l) - f2, 0.0))) / (2.0 * v_l[0]));
  f1 = gm * v_r[4];
  f2 = 4.0 * f1 * (v_r[5] * v_r[5]);
  double vf_r = sqrt(((f1 + b2_r) + sqrt(fmx((f1 + b2_r) * (f1 + b2_r) - f2, 0.0))) / (2.0 * v_r[0]));

  double sl = fmn(v_l[1], v_r[1]) - fmx(vf_l, vf_r);
  double sr = fmx(v_l[1], v_r[1]) + fmx(vf_l, vf_r);

  if (sl >= 0.0) {
    for (int n = 0; n < 8; ++n) flx[n] = flx_l[n];
  } else if (sr <= 0.0) {
    for (int n = 0; n < 8; ++n) flx[n] = flx_r[n];
  } else {
    f1 = 1.0 / (sr - sl);
    for (int n = 0; n < 8; ++n) u_hll[n] = f1 * (sr * u_r[n] - sl * u_l[n] - flx_r[n] + flx_l[n]);
    double sm = u_hll[1] / u_hll[0];
    double pt = pt_l + v_l[0] * (sl - v_l[1]) * (sm - v_l[1]);
    double ro_l1 = v_l[0] * (sl - v_l[1]) / (sl - sm);
    double ro_r1 = v_r[0] * (sr - v_r[1]) / (sr - sm);
    double sal = fabs(u_hll[5]) / sqrt(ro_l1);
    double sar = fabs(u_hll[5]) / sqrt(ro_r1);

    if ((sl >= (sm - HLLG_FACTOR * sal)) || ((sm + HLLG_FACTOR * sar) >= sr)) {
      /* revert to HLLC-G */
      double vy_2 = u_hll[2] / u_hll[0];
      double vz_2 = u_hll[3] / u_hll[0];
      if (sm >= 0.0) {
        u2[4] = ((sl - v_l[1]) * u_l[4] - pt_l * v_l[1] + pt * sm +
                 u_hll[5] * (vbL - sm * u_hll[5] - vy_2 * u_hll[6] - vz_2 * u_hll[7])) /
                (sl - sm);
        u2[1] = ro_l1 * sm;
        u2[2] = ro_l1 * vy_2;
        u2[3] = ro_l1 * vz_2;
        flx[0] = sl * (ro_l1 - v_l[0]) + flx_l[0];
        for (int n = 1; n < 5; ++n) flx[n] = sl * (u2[n] - u_l[n]) + flx_l[n];
        for (int n = 5; n < 8; ++n) flx[n] = sl * (u_hll[n] - v_l[n]) + flx_l[n];
      } else {
        u2[4] = ((sr - v_r[1]) * u_r[4] - pt_r * v_r[1] + pt * sm +
                 u_hll[5] * (vbR - sm * u_hll[5] - vy_2 * u_hll[6] - vz_2 * u_hll[7])) /
                (sr - sm);
        u2[1] = ro_r1 * sm;
        u2[2] = ro_r1 * vy_2;
        u2[3] = ro_r1 * vz_2;
        flx[0] = sr * (ro_r1 - v_r[0]) + flx_r[0];
        for (int n = 1; n < 5; ++n) flx[n] = sr * (u2[n] - u_r[n]) + flx_r[n];
        for (int n = 5; n < 8; ++n) flx[n] = sr * (u_hll[n] - v_r[n]) + flx_r[n];
      }
    } else {
      /* intermediate state (L*) */
      f1 = 1.0 / (v_l[0] * (sl - v_l[1]) * (sl - sm) - u_hll[5] * u_hll[5]);
      u_l1[5] = u_hll[5];
      u_l1[6] = v_l[6] * f1 * (v_l[0] * ((sl - v_l[1]) * (sl - v_l[1])) - u_hll[5] * u_hll[5]);
      u_l1[7] = v_l[7] * f1 * (v_l[0] * ((sl - v_l[1]) * (sl - v_l[1])) - u_hll[5] * u_hll[5]);
      double vy_l1 = v_l[2] - f1 * u_hll[5] * v_l[6] * (sm - v_l[1]);
      double vz_l1 = v_l[3] - f1 * u_hll[5] * v_l[7] * (sm - v_l[1]);
      u_l1[0] = ro_l1;
      u_l1[4] = ((sl - v_l[1]) * u_l[4] - pt_l * v_l[1] + pt * sm +
                 u_hll[5] * (vbL - sm * u_hll[5] - vy_l1 * u_l1[6] - vz_l1 * u_l1[7])) /
                (sl - sm);
      u_l1[1] = ro_l1 * sm;
      u_l1[2] = ro_l1 * vy_l1;
      u_l1[3] = ro_l1 * vz_l1;

      /* intermediate state (R*) */
      f1 = 1.0 / (v_r[0] * (sr - v_r[1]) * (sr - sm) - u_hll[5] * u_hll[5]);
      u_r1[5] = u_hll[5];
      u_r1[6] = v_r[6] * f1 * (v_r[0] * ((sr - v_r[1]) * (sr - v_r[1])) - u_hll[5] * u_hll[5]);
      u_r1[7] = v_r[7] * f1 * (v_r[0] * ((sr - v_r[1]) * (sr - v_r[1])) - u_hll[5] * u_hll[5]);
      double vy_r1 = v_r[2] - f1 * u_hll[5] * v_r[6] * (sm - v_r[1]);
      double vz_r1 = v_r[3] - f1 * u_hll[5] * v_r[7] * (sm - v_r[1]);
      u_r1[0] = ro_r1;
      u_r1[4] = ((sr - v_r[1]) * u_r[4] - pt_r * v_r[1] + pt * sm +
                 u_hll[5] * (vbR - sm * u_hll[5] - vy_r1 * u_r1[6] - vz_r1 * u_r1[7])) /
                (sr - sm);
      u_r1[1] = ro_r1 * sm;
      u_r1[2] = ro_r1 * vy_r1;
      u_r1[3] = ro_r1 * vz_r1;

      /* rotational discontinuities */
      double sl1 = sm - sal;
      double sr1 = sm + sar;
      if (sl1 >= 0.0) {
        flx[0] = sl * (u_l1[0] - v_l[0]) + flx_l[0];
        for (int n = 1; n < 5; ++n) flx[n] = sl * (u_l1[n] - u_l[n]) + flx_l[n];
        for (int n = 5; n < 8; ++n) flx[n] = sl * (u_l1[n] - v_l[n]) + flx_l[n];
      } else if (sr1 <= 0.0) {
        flx[0] = sr * (u_r1[0] - v_r[0]) + flx_r[0];
        for (int n = 1; n < 5; ++n) flx[n] = sr * (u_r1[n] - u_r[n]) + flx_r[n];
        for (int n = 5; n < 8; ++n) flx[n] = sr * (u_r1[n] - v_r[n]) + flx_r[n];
      } else {
        /* central states */
        double ro_ls = sqrt(ro_l1);
        double ro_rs = sqrt(ro_r1);
        f1 = 1.0 / (ro_ls + ro_rs);
        f2 = copysign(1.0, u_hll[5]);
        double vy_2 = f1 * (ro_ls * vy_l1 + ro_rs * vy_r1 + (u_r1[6] - u_l1[6]) * f2);
        double vz_2 = f1 * (ro_ls * vz_l1 + ro_rs * vz_r1 + (u_r1[7] - u_l1[7]) * f2);
        u2[5] = u_hll[5];
        u2[6] = f1 * (ro_ls * u_r1[6] + ro_rs * u_l1[6] + ro_ls * ro_rs * (vy_r1 - vy_l1) * f2);
        u2[7] = f1 * (ro_ls * u_r1[7] + ro_rs * u_l1[7] + ro_ls * ro_rs * (vz_r1 - vz_l1) * f2);
        if (sm >= 0.0) {
          u2[0] = ro_l1;
          u2[4] = u_l1[4] - ro_ls * (vy_l1 * u_l1[6] + vz_l1 * u_l1[7] - vy_2 * u2[6] - vz_2 * u2[7]) * f2;
          u2[1] = ro_l1 * sm;
          u2[2] = ro_l1 * vy_2;
          u2[3] = ro_l1 * vz_2;
          flx[0] = sl1 * u2[0] - (sl1 - sl) * u_l1[0] - sl * v_l[0] + flx_l[0];
          for (int n = 1; n < 5; ++n) flx[n] = sl1 * u2[n] - (sl1 - sl) * u_l1[n] - sl * u_l[n] + flx_l[n];
          for (int n = 5; n < 8; ++n) flx[n] = sl1 * u2[n] - (sl1 - sl) * u_l1[n] - sl * v_l[n] + flx_l[n];
        } else {
          u2[0] = ro_r1;
          u2[4] = u_r1[4] + ro_rs * (vy_r1 * u_r1[6] + vz_r1 * u_r1[7] - vy_2 * u2[6] - vz_2 * u2[7]) * f2;
          u2[1] = ro_r1 * sm;
          u2[2] = ro_r1 * vy_2;
          u2[3] = ro_r1 * vz_2;
          flx[0] = sr1 * u2[0] - (sr1 - sr) * u_r1[0] - sr * v_r[0] + flx_r[0];
          for (int n = 1; n < 5; ++n) flx[n] = sr1 * u2[n] - (sr1 - sr) * u_r1[n] - sr * u_r[n] + flx_r[n];
          for (int n = 5; n < 8; ++n) flx[n] = sr1 * u2[n] - (sr1 - sr) * u_r1[n] - sr * v_r[n] + flx_r[n];
        }
      }
    }
  }
  if (divb) {
    double ch = cmax;
    flx[5] = 0.5 * (u_l[8] + u_r[8] - ch * (v_r[5] - v_l[5]));
    flx[8] = 0.5 * (ch * ch * (v_l[5] + v_r[5]) - ch * (v_r[8] - v_l[8]));
  }
}

/* Component permutations of set_HLLC_fluxes / set_HLLD_fluxes (HLL_rot.f90:295-461):
 * direction 2 swaps (vx,vy) and (bx,by); direction 3 swaps (vx,vz) and (bx,bz). */
static const int PERM_H[3][5] = {{0, 1, 2, 3, 4}, {0, 2, 1, 3, 4}, {0, 3, 2, 1, 4}};
static const int PERM_M[3][9] = {{0, 1, 2, 3, 4, 5, 6, 7, 8},
                                 {0, 2, 1, 3, 4, 6, 5, 7, 8},
                                 {0, 3, 2, 1, 4, 7, 6, 5, 8}};

/* set_HLLC_fluxes / set_HLLD_fluxes for one direction: F(.., n) of the face between
 * s and s+1 along dir, for s = 0..len-2 and every cell of the other axes. */
static void set_fluxes(const orc_ctx *c, double *F, const double *VL, const double *VR, int dir,
                       int mhd) {
  int ix = c->ix, jx = c->jx, kx = c->kx;
  size_t nc = c->nc;
  int nvar = mhd ? c->nm : c->nh;
  int ie = dir == 1 ? ix - 1 : ix, je = dir == 2 ? jx - 1 : jx, ke = dir == 3 ? kx - 1 : kx;
  const int *perm = mhd ? PERM_M[dir - 1] : PERM_H[dir - 1];
  int divb = c->p.flag_divb == 1;
  double gm = c->p.gm, cmax = c->cmax;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < ke; ++k)
    for (int j = 0; j < je; ++j)
      for (int i = 0; i < ie; ++i) {
        double vl[9], vr[9], fl[9];
        size_t q = AT(c, i, j, k);
        for (int n = 0; n < nvar; ++n) {
          vl[n] = VL[q + perm[n] * nc];
          vr[n] = VR[q + perm[n] * nc];
        }
        if (mhd) hlld_flux(vl, vr, fl, nvar, gm, divb, cmax);
        else hllc_flux(vl, vr, fl, gm);
        for (int n = 0; n < nvar; ++n) F[q + perm[n] * nc] = fl[n];
      }
}

/* get_rotation (Util_rot.f90:148-236), s_order 2 branch, of B = U_m(:,:,:,6:8): the
 * central-difference curl on cells 2..ix-1 (2..jx-1), zero elsewhere. */
static void get_rotation(const orc_ctx *c, double *R) {
  size_t nc = c->nc;
  const double *bx = c->U_m + 5 * nc, *by = c->U_m + 6 * nc, *bz = c->U_m + 7 * nc;
  int ix = c->ix, jx = c->jx;
  memset(R, 0, sizeof(double) * 3 * nc);
  double *R1 = R, *R2 = R + nc, *R3 = R + 2 * nc;
  if (c->p.ndim == 1) {
    for (int j = 0; j < jx; ++j)
      for (int i = 1; i < ix - 1; ++i) {
        size_t q = AT(c, i, j, 0);
        R2[q] = -(bz[q + 1] - bz[q - 1]) / (2.0 * c->dx[i]);
        R3[q] = (by[q + 1] - by[q - 1]) / (2.0 * c->dx[i]);
      }
    return;
  }
#pragma omp parallel for schedule(static)
  for (int j = 1; j < jx - 1; ++j)
    for (int i = 1; i < ix - 1; ++i) {
      size_t q = AT(c, i, j, 0), s = (size_t)ix;
      R1[q] = (bz[q + s] - bz[q - s]) / (2.0 * c->dy[j]);
      R2[q] = -(bz[q + 1] - bz[q - 1]) / (2.0 * c->dx[i]);
      R3[q] = ((by[q + 1] - by[q - 1]) / (2.0 * c->dx[i]) - (bx[q + s] - bx[q - s]) / (2.0 * c->dy[j]));
    }
}

/* resistive_flux (Solver_rot.f90:505-638), flag_sch=0 branch, for direction dir: E =
 * eta*curl B at the cells, averaged onto the faces 1..ix-1 (1..jx-1) and added to the
 * energy and induction fluxes. */
static void resistive_flux(orc_ctx *c, int dir, double *F) {
  size_t nc = c->nc;
  int ix = c->ix, jx = c->jx;
  double *w = malloc(sizeof(double) * 6 * nc);
  double *cur = w, *ex = w + 3 * nc, *ey = w + 4 * nc, *ez = w + 5 * nc;
  get_rotation(c, cur);
  for (size_t q = 0; q < nc; ++q) {
    ex[q] = cur[q] * c->eta[q];
    ey[q] = cur[q + nc] * c->eta[q];
    ez[q] = cur[q + 2 * nc] * c->eta[q];
  }
  const double *bx = c->U_m + 5 * nc, *by = c->U_m + 6 * nc, *bz = c->U_m + 7 * nc;
  if (dir == 1) {
    for (int j = 0; j < jx; ++j)
      for (int i = 0; i < ix - 1; ++i) {
        size_t q = AT(c, i, j, 0), r = q + 1;
        F[q + 4 * nc] = F[q + 4 * nc] +
                        0.25 * ((ey[r] + ey[q]) * (bz[q] + bz[r]) - (ez[q] + ez[r]) * (by[q] + by[r]));
        F[q + 6 * nc] = F[q + 6 * nc] - 0.5 * (ez[q] + ez[r]);
        F[q + 7 * nc] = F[q + 7 * nc] + 0.5 * (ey[q] + ey[r]);
      }
  } else if (dir == 2) {
    for (int j = 0; j < jx - 1; ++j)
      for (int i = 0; i < ix; ++i) {
        size_t q = AT(c, i, j, 0), r = q + (size_t)ix;
        F[q + 4 * nc] = F[q + 4 * nc] +
                        0.25 * ((ez[r] + ez[q]) * (bx[q] + bx[r]) - (ex[q] + ex[r]) * (bz[q] + bz[r]));
        F[q + 5 * nc] = F[q + 5 * nc] + 0.5 * (ez[q] + ez[r]);
        F[q + 7 * nc] = F[q + 7 * nc] - 0.5 * (ex[q] + ex[r]);
      }
  }
  free(w);
}

/* set_resistivity resi_type 2 and 3 (Res_rot.f90:37-60): eta from |curl B| of the current
 * state (get_rotation of U_m(:,:,:,6:8), zero on the outermost layer): type 2 eta_0, or
 * 11 eta_0 where |curl B| >= j_cri; type 3 eta_0 (vd/vd_cri - 1)**2 where the drift
 * vd = |curl B|/rho_i >= vd_cri, else 0. */
static void set_resistivity_anomalous(orc_ctx *c) {
  const pip_params *p = &c->p;
  size_t nc = c->nc;
  double *cur = malloc(sizeof(double) * 3 * nc);
  get_rotation(c, cur);
  const double *r1 = cur, *r2 = cur + nc, *r3 = cur + 2 * nc;
  for (size_t q = 0; q < nc; ++q) {
    double c2 = sqrt(r1[q] * r1[q] + r2[q] * r2[q] + r3[q] * r3[q]);
    if (p->resi_type == 2) {
      c->eta[q] = p->eta_0;
      if (c2 >= p->j_cri) c->eta[q] = p->eta_0 * 11.0;
    } else {
      double vdri = c2 / c->U_m[q];
      c->eta[q] = 0.0;
      if (vdri >= p->vd_cri) {
        double a = vdri / p->vd_cri - 1.0;
        c->eta[q] = p->eta_0 * (a * a);
      }
    }
  }
  free(cur);
}

void orc_resistivity(orc_ctx *c, double *eta) {
  ensure_coefficients(c);
  memcpy(eta, c->eta, sizeof(double) * c->nc);
}

void orc_set_resistivity(orc_ctx *c, const double *eta) {
  if (c->eta) memcpy(c->eta, eta, sizeof(double) * c->nc);
}

/* hlld_fluxes_ideal / hllc_fluxes_ideal for one direction (HLL_rot.f90:94-121), then
 * set_flux's resistive_flux (Solver_rot.f90:155-156). */
static void flux_dir(orc_ctx *c, int dir, double *F_h, double *F_m) {
  size_t nc = c->nc;
  double *V = malloc(sizeof(double) * nc * 9);
  double *VL = malloc(sizeof(double) * nc * 9);
  double *VR = malloc(sizeof(double) * nc * 9);
  u2v_mhd(c, c->U_m, V);
  get_side(c, V, VL, VR, dir, c->nm);
  set_fluxes(c, F_m, VL, VR, dir, 1);
  if (c->resi) resistive_flux(c, dir, F_m);
  u2v_hd(c, c->U_h, V);
  get_side(c, V, VL, VR, dir, c->nh);
  set_fluxes(c, F_h, VL, VR, dir, 0);
  free(V); free(VL); free(VR);
}

void orc_flux(orc_ctx *c, int dir, double *F_h, double *F_m) {
  ensure_coefficients(c);
  memset(F_h, 0, sizeof(double) * c->nc * c->nh);
  memset(F_m, 0, sizeof(double) * c->nc * c->nm);
  flux_dir(c, dir, F_h, F_m);
}

/* ---------------------------------------------------------------- sources */

/* Ionisation/recombination rates of PIP_IR_POWERLAW (a new law) from the ion state U_m:
 * pressure by get_Pr_MHD's expression and floor (Scheme_rot.f90:112-121, without its
 * energy rewrite), temperature by get_Te_MHD (:104-110), Te = 0.5*gm*(pr/ro). */
static void set_ir_rates(orc_ctx *c) {
  size_t nc = c->nc;
  double gm = c->p.gm, pr_lim = c->p.pr_lim;
  const double *U = c->U_m;
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < nc; ++q) {
    double u1 = U[q], u2 = U[q + nc], u3 = U[q + 2 * nc], u4 = U[q + 3 * nc];
    double u6 = U[q + 5 * nc], u7 = U[q + 6 * nc], u8 = U[q + 7 * nc];
    double pr = (gm - 1.0) * (U[q + 4 * nc] -
                              0.5 * ((u2 * u2 + u3 * u3 + u4 * u4) / u1 + u6 * u6 + u7 * u7 + u8 * u8));
    pr = fmx(pr, pr_lim);
    double te = 0.5 * gm * (pr / u1);
    double rs = 1.0 / sqrt(te);
    c->gm_rec[q] = c->p.ir_rec_coef * rs;
    c->gm_ion[q] = c->p.ir_ion_coef * rs * exp(-c->p.ir_chi / te);
  }
}

/* alpha_c of set_collisional's col_type 1..6 (PIP_rot.f90:53-95) for one cell from the two
 * temperatures and the drift, with the Fortran operation order (left to right). */
static double alpha_c_cell(int type, double col, double beta, double gm, double te_h, double te_m,
                           double vdx, double vdy, double vdz) {
  double T = te_h + te_m;
  double a = col * sqrt(T / 2.0);
  if (type == 1) return a / sqrt(beta / 2.0 * gm);
  if (type == 2) return a;
  double v2 = vdx * vdx + vdy * vdy + vdz * vdz;     /* sum(vd**2,dim=4) */
  a = a * sqrt(1.0 + 9.0 * PI_REF / 64.0 * gm / 2.0 * v2 / T);
  if (type == 3) return a / sqrt(beta / 2.0 * gm);
  if (type == 4) return a;
  if (type == 5)
    return a / sqrt(beta / 2.0 * gm) * pow((beta / 2.0 * gm) / T / 2.0 + gm * PI_REF / 16.0 * v2, 0.125);
  return a / pow(T / 2.0 + gm * PI_REF / 16.0 * v2, 0.125);
}

/* set_collisional for col_type >= 1 (PIP_rot.f90:44-97): get_Te_MHD and get_Te_HD
 * (Scheme_rot.f90:83-128) rewrite both energies through the floored pressure and give
 * Te_m = 0.5*gm*pr/ro, Te_h = gm*pr/ro; get_vel_diff (:988-999) gives the drift; alpha_c of
 * every cell, ghosts included, goes to c->ac.  The floor `if(minval(pr).le.pr_lim)
 * pr=max(pr,pr_lim)` is the per-cell max. */
/* get_Te_MHD and get_Te_HD (Scheme_rot.f90:83-128) on cell q: both energies rewritten
 * through the floored pressure; Te_m = 0.5*gm*pr/ro, Te_h = gm*pr/ro. */
static void get_te_cell(orc_ctx *c, size_t q, double *te_m, double *te_h) {
  size_t nc = c->nc;
  double gm = c->p.gm, pr_lim = c->p.pr_lim;
  double *Um = c->U_m, *Uh = c->U_h;
  double m1 = Um[q], m2 = Um[q + nc], m3 = Um[q + 2 * nc], m4 = Um[q + 3 * nc];
  double m6 = Um[q + 5 * nc], m7 = Um[q + 6 * nc], m8 = Um[q + 7 * nc];
  double prm = (gm - 1.0) * (Um[q + 4 * nc] -
                             0.5 * ((m2 * m2 + m3 * m3 + m4 * m4) / m1 + m6 * m6 + m7 * m7 + m8 * m8));
  prm = fmx(prm, pr_lim);
  Um[q + 4 * nc] = prm / (gm - 1.0) + 0.5 * ((m2 * m2 + m3 * m3 + m4 * m4) / m1 + m6 * m6 +
                                             m7 * m7 + m8 * m8);
  *te_m = 0.5 * gm * (prm / m1);
  double h1 = Uh[q], h2 = Uh[q + nc], h3 = Uh[q + 2 * nc], h4 = Uh[q + 3 * nc];
  double prh = (gm - 1.0) * (Uh[q + 4 * nc] - 0.5 * (h2 * h2 + h3 * h3 + h4 * h4) / h1);
  prh = fmx(prh, pr_lim);
  Uh[q + 4 * nc] = prh / (gm - 1.0) + 0.5 * ((h2 * h2 + h3 * h3 + h4 * h4) / h1);
  *te_h = gm * (prh / h1);
}

static void set_collisional(orc_ctx *c) {
  const pip_params *p = &c->p;
  size_t nc = c->nc;
  double gm = p->gm, col = p->col, beta = p->beta;
  int type = c->col_type;
  const double *Um = c->U_m, *Uh = c->U_h;
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < nc; ++q) {
    double te_m, te_h;
    get_te_cell(c, q, &te_m, &te_h);
    double m1 = Um[q], m2 = Um[q + nc], m3 = Um[q + 2 * nc], m4 = Um[q + 3 * nc];
    double h1 = Uh[q], h2 = Uh[q + nc], h3 = Uh[q + 2 * nc], h4 = Uh[q + 3 * nc];
    c->ac[q] = alpha_c_cell(type, col, beta, gm, te_h, te_m, h2 / h1 - m2 / m1, h3 / h1 - m3 / m1,
                            h4 / h1 - m4 / m1);
  }
}

/* ---------------------------------------------------------------- 6-level hydrogen model */

/* Literals the Fortran writes without a d0 exponent are default reals: rounded to float
 * first (kboltz, melec, a0bohr of get_col_ion_coeff, PIP_rot.f90:366-369; 2.18e-18 of
 * :383; 1.0e14 of :591; 1.e-16 of :1138; Eev of IRgetionpot :1170; 8.6173e-5 of :1224). */
#define NL_KB ((double)1.38064852e-23f)
#define NL_ME ((double)9.10938356e-31f)
#define NL_A0 ((double)5.29e-11f)
#define NL_EJ ((double)2.18e-18f)
#define NL_E14 ((double)1.0e14f)
#define NL_FLOOR ((double)1.e-16f)
#define NL_EVK ((double)8.6173e-5f)
#define NL_KBHAT 1.38064852
#define NL_MEHAT 9.10938356
#define NL_HHAT 6.62607004

/* colexpintcalc.f90's ionexpfittest: trapezoid sums of exp(-z*t)*t**(-istar) from t = 1 in
 * steps of 0.001 until a step adds no more than 1e-4 of the first. */
static double nl_expint_trap(double zhat, double istar) {
  const double stepsize = 0.001, tol = 0.0001;
  double a = 1.0, b = a + stepsize;
  double fa = exp(-zhat * a) * pow(a, -istar), fb = exp(-zhat * b) * pow(b, -istar);
  double sol0 = 0.5 * (b - a) * (fa + fb), sol = sol0, dif = 1.0;
  while (dif > tol) {
    a = b;
    b = a + stepsize;
    fa = exp(-zhat * a) * pow(a, -istar);
    fb = exp(-zhat * b) * pow(b, -istar);
    double solt = 0.5 * (b - a) * (fa + fb);
    sol = sol + solt;
    dif = solt / sol0;
  }
  return sol;
}

/* colexpintcalc.f90 (the generator of expintcalc/colexp.dat, which expintread loads,
 * PIP_rot.f90:315-333): nsamps+1 rows (yn, E0(yn), E1(yn), E2(yn)) for
 * yn = ymin + t*(108 - ymin)/nsamps; out is column-major (4, nsamps+1). */
void orc_expint_table(long nsamps, double *out) {
  const double ymin = 0.54 / 13.6 * NL_EJ / NL_KB / 100000.0, ymax = 108.0;
  const double dy = (ymax - ymin) / (double)nsamps;
#pragma omp parallel for schedule(dynamic, 64)
  for (long t = 0; t <= nsamps; ++t) {
    double yn = ymin + (double)t * dy;
    out[4 * t] = yn;
    out[4 * t + 1] = nl_expint_trap(yn, 0.0);
    out[4 * t + 2] = nl_expint_trap(yn, 1.0);
    out[4 * t + 3] = nl_expint_trap(yn, 2.0);
  }
}

/* The cell-independent part of get_col_ion_coeff (PIP_rot.f90:378-439, 507-524), in the
 * Fortran operation order. */
static void nl_constants(orc_ctx *c) {
  static const double ev[6] = {13.6, 3.4, 1.51, 0.85, 0.54, 0.0};
  static const double gw[6] = {2.0, 8.0, 18.0, 32.0, 50.0, 1.0};
  for (int k = 0; k < 6; ++k) {
    double n = (double)(k + 1);
    c->nk.gw[k] = gw[k];
    c->nk.eion[k] = ev[k] / 13.6 * NL_EJ;
    c->nk.rn[k] = k == 0 ? 0.45 : 1.94 * pow(n, -1.57);
    c->nk.bn[k] = k == 0 ? -0.603
                         : (1.0 / n) * (4.0 - 18.63 / n + 36.24 / (n * n) - 28.09 / (n * n * n));
  }
  const double pi = PI_REF;
  for (int a = 0; a < 5; ++a) {
    double ri = (double)(a + 1);
    for (int b = a + 1; b < 5; ++b) {
      double rj = (double)(b + 1), r = ri / rj;
      double x = 1.0 - r * r;
      double g;
      if (a == 0) g = 1.1330 - 0.4059 / x + 0.07014 / (x * x);
      else if (a == 1) g = 1.0785 - 0.2319 / x + 0.02947 / (x * x);
      else
        g = 0.9935 + 0.2328 / ri - 0.1296 / (ri * ri) -
            (1.0 / x) * (1.0 / ri) * (0.6282 - 0.5598 / ri + 0.5299 / (ri * ri)) +
            (1.0 / x) * (1.0 / x) * (1.0 / (ri * ri)) * (0.3887 - 1.181 / ri + 1.470 / (ri * ri));
      double fnn = 32.0 / 3.0 / sqrt(3.0) / pi * ri / (rj * rj * rj) / (x * x * x) * g;
      c->nk.xrat[a][b] = x;
      c->nk.enn[a][b] = c->nk.eion[a] - c->nk.eion[b];
      c->nk.rnn[a][b] = c->nk.rn[a] * x;
      c->nk.ann[a][b] = 2.0 * (ri * ri) / x * fnn;
      c->nk.bnn[a][b] = 4.0 * ((ri * ri) * (ri * ri)) / (rj * rj * rj) / (x * x) *
                        (1.0 + 4.0 / 3.0 / x + c->nk.bn[a] / (x * x));
      c->nk.lgt[a][b] = log(2.0 * (ri * ri) / x);
    }
    double g1, g2, g3;
    if (a == 0) { g1 = 1.1330; g2 = -0.4059; g3 = 0.07014; }
    else if (a == 1) { g1 = 1.0785; g2 = -0.2319; g3 = 0.02947; }
    else {
      g1 = 0.9935 + 0.2328 / ri - 0.1296 / (ri * ri);
      g2 = (-1.0 / ri) * (0.6282 - 0.5598 / ri + 0.5299 / (ri * ri));
      g3 = (1.0 / ri) * (1.0 / ri) * (0.3887 - 1.181 / ri + 1.470 / (ri * ri));
    }
    c->nk.an0[a] = 32.0 / 3.0 / sqrt(3.0) / pi * ri + g1 / 3.0 + g2 / 4.0 + g3 / 5.0;
    c->nk.bn0[a] = 2.0 / 3.0 * (ri * ri) * (5.0 + c->nk.bn[a]);
    c->nk.lgi[a] = log(2.0 * (ri * ri));
  }
}

/* ionexpfitinterp2 with rad = 0 (PIP_rot.f90:919-946): quadratic interpolation of E_i at z
 * through table rows xindex..xindex+2.  The reference clamps xindex to 1..n-1 and then reads
 * row n+1 at the top end, past its table; here xindex stops at n-2. */
static double nl_interp(const orc_ctx *c, double z, int i) {
  const double *t = c->etab;
  long n = c->netab;
  double xmin = t[0], xmax = t[4 * (n - 1)], xrange = xmax - xmin;
  double f = floor((z - xmin) / xrange * (double)n);
  long xi;
  if (!(f > 0.0)) xi = 1;
  else if (f >= (double)n) xi = n - 1;
  else xi = (long)f;
  if (xi > n - 2) xi = n - 2;
  const double *r0 = t + 4 * (xi - 1), *r1 = r0 + 4, *r2 = r0 + 8;
  double x0 = r0[0], x1 = r1[0], x2 = r2[0];
  double w0 = ((z - x1) * (z - x2)) / ((x0 - x1) * (x0 - x2));
  double w1 = ((z - x0) * (z - x2)) / ((x1 - x0) * (x1 - x2));
  double w2 = ((z - x0) * (z - x1)) / ((x2 - x0) * (x2 - x1));
  return w0 * r0[i + 1] + w1 * r1[i + 1] + w2 * r2[i + 1];
}

/* get_col_ion_coeff (PIP_rot.f90:361-616) for one cell of electron temperature te [K] and
 * density ne: colrat (6x6, cr[a*6+b] = colrat(a+1,b+1)) and the unnormalised sums
 * gi = sum max(Nexcite(ii)*colrat(ii,6),0), gr = sum max(Nexcite(6)*colrat(6,ii),0).
 * Returns 1 where the reference would stop on a negative rate. */
static int nl_cell(const orc_ctx *c, double te, double ne, const double *nx, double *cr,
                   double *gi, double *gr) {
  const double pi = PI_REF;
  double colex[5][6];
  int bad = 0;
  double s = sqrt(8.0 * NL_KB * te / pi / NL_ME);
  for (int a = 0; a < 5; ++a) {
    double ri = (double)(a + 1);
    for (int b = a + 1; b < 5; ++b) {
      double yhat = c->nk.enn[a][b] / NL_KB / te;
      double zhat = c->nk.rnn[a][b] + c->nk.enn[a][b] / NL_KB / te;
      double E1y = nl_interp(c, yhat, 1), E1z = nl_interp(c, zhat, 1);
      double E2y = nl_interp(c, yhat, 2), E2z = nl_interp(c, zhat, 2);
      double ann = c->nk.ann[a][b];
      colex[a][b] = ne * s * 2.0 * (ri * ri) / c->nk.xrat[a][b] * pi * (NL_A0 * NL_A0) *
                    (yhat * yhat) *
                    (ann * ((1.0 / yhat + 0.5) * E1y - (1.0 / zhat + 0.5) * E1z) +
                     (c->nk.bnn[a][b] - ann * c->nk.lgt[a][b]) * (E2y / yhat - E2z / zhat));
    }
    double yn = c->nk.eion[a] / NL_KB / te;
    double zn = c->nk.rn[a] + c->nk.eion[a] / NL_KB / te;
    double E1y = nl_interp(c, yn, 1), E1z = nl_interp(c, zn, 1);
    double E2y = nl_interp(c, yn, 2), E2z = nl_interp(c, zn, 2);
    double E0y = nl_interp(c, yn, 0), E0z = nl_interp(c, zn, 0);
    double ziyn = E0y - 2.0 * E1y + E2y, zizn = E0z - 2.0 * E1z + E2z;
    double an0 = c->nk.an0[a];
    colex[a][5] = ne * s * 2.0 * (ri * ri) * pi * (NL_A0 * NL_A0) * (yn * yn) *
                  (an0 * (E1y / yn - E1z / zn) + (c->nk.bn0[a] - an0 * c->nk.lgi[a]) * (ziyn - zizn));
    if (colex[a][5] < 0.0) bad = 1;
  }
  for (int k = 0; k < 36; ++k) cr[k] = 0.0;
  for (int a = 0; a < 5; ++a) {
    for (int b = 0; b < 5; ++b) {
      if (a == b) cr[a * 6 + b] = 0.0;
      else if (b > a) cr[a * 6 + b] = c->nk.gw[a] / c->nk.gw[b] * colex[a][b];
      else cr[a * 6 + b] = colex[b][a] * exp(-((c->nk.eion[b] - c->nk.eion[a]) / NL_KB / te));
    }
    cr[a * 6 + 5] = colex[a][5] * exp(-((c->nk.eion[5] - c->nk.eion[a]) / NL_KB / te));
  }
  for (int a = 0; a < 5; ++a)
    cr[30 + a] = ne * cr[a * 6 + 5] * c->nk.gw[a] / c->nk.gw[5] / 2.0 *
                 pow(2.0 * pi * NL_MEHAT * NL_KBHAT * te / NL_HHAT / NL_HHAT * NL_E14, -3.0 / 2.0) *
                 exp(c->nk.eion[a] / NL_KB / te);
  for (int k = 0; k < 36; ++k)
    if (cr[k] < 0.0) bad = 1;
  double si = 0.0, sr = 0.0;
  for (int a = 0; a < 5; ++a) {
    si = si + fmx(nx[a] * cr[a * 6 + 5], 0.0);
    sr = sr + fmx(nx[5] * cr[30 + a], 0.0);
  }
  *gi = si;
  *gr = sr;
  return bad;
}

/* tfac of set_IR type 4 (PIP_rot.f90:240-248); 5.0/3.0 is a default-real quotient there. */
static double nl_tfac(const orc_ctx *c) {
  const pip_params *p = &c->p;
  if (p->flag_col % 2 == 1) return p->t_norm / ((double)(5.0f / 3.0f) * c->f_p_p_ini / c->f_p_ini);
  return p->beta / 2.0 * c->f_p_p_ini * 5.0 / 6.0 / c->f_p_ini;
}

/* IRgetionpot (PIP_rot.f90:1162-1235) on cell q from colrat cr and populations nx. */
static double nl_ionpot(const orc_ctx *c, const double *cr, const double *nx) {
  static const float eevf[6] = {13.6f, 3.4f, 1.51f, 0.85f, 0.54f, 0.0f};
  double eev[6];
  for (int k = 0; k < 6; ++k) eev[k] = (double)eevf[k];
  double il = 0.0, ig = 0.0;
  for (int i = 0; i < 5; ++i) {
    il = il + cr[i * 6 + 5] * eev[i] * nx[i];
    ig = ig + cr[30 + i] * eev[i] * nx[5];
    for (int j = 1; j < 5; ++j) {
      il = il + nx[i] * cr[i * 6 + j] * (eev[i] - eev[j]);
      ig = ig + nx[j] * (cr[j * 6 + i] * (eev[i] - eev[j]));
    }
  }
  const pip_params *p = &c->p;
  double en;
  if (p->flag_col % 2 == 1) en = (il - ig) / p->gm / p->t_norm / NL_EVK;
  else en = (il - ig) / (p->beta / p->t_norm / 2.0 / NL_EVK);
  return en / c->gm_rec_ref * p->t_ir;
}

/* set_IR type 4 (PIP_rot.f90:232-296): get_Te_HD/get_Te_MHD rewrite both energies; on the
 * first call of a fresh run (the prologue's, :250-280) Gm_rec_ref from the rates at
 * (T_norm, n_norm) with cell (1,1,1)'s populations and ion_pot from those rates; then
 * colrat of every cell from Te_p*T0/tfac and U_m(1)*n0/n0fac, and the normalised rates. */
static void set_ir_nlevel(orc_ctx *c) {
  const pip_params *p = &c->p;
  size_t nc = c->nc;
  if (!c->etab) {
    c->nlev_bad = 1;   /* no table: orc_set_nlevel was not called */
    return;
  }
  double T0 = p->t_norm, n0 = p->n_norm, tfac = nl_tfac(c);
  double *te = malloc(sizeof(double) * nc);
  for (size_t q = 0; q < nc; ++q) {
    double te_n;
    get_te_cell(c, q, &te[q], &te_n);
  }
  if (!c->nlev_init) {
    double nx0[6], cr[36], gi, gr;
    for (int k = 0; k < 6; ++k) nx0[k] = c->nex[k * nc];
    nl_cell(c, T0, n0, nx0, cr, &gi, &gr);
    c->gm_rec_ref = gr;
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < nc; ++q) {
      double nx[6];
      for (int k = 0; k < 6; ++k) nx[k] = c->nex[q + k * nc];
      c->ion_pot[q] = nl_ionpot(c, cr, nx);
    }
    c->nlev_init = 1;
  }
  const double *Uh = c->U_h, *Um = c->U_m;
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
  for (size_t q = 0; q < nc; ++q) {
    double nx[6], cr[36], gi, gr;
    for (int k = 0; k < 6; ++k) nx[k] = c->nex[q + k * nc];
    bad |= nl_cell(c, te[q] * T0 / tfac, Um[q] * n0 / c->n0fac, nx, cr, &gi, &gr);
    for (int k = 0; k < 36; ++k) c->colrat[q + k * nc] = cr[(k % 6) * 6 + k / 6];
    c->gm_ion[q] = gi / Uh[q] / c->gm_rec_ref * p->t_ir;
    c->gm_rec[q] = gr / Um[q] / c->gm_rec_ref * p->t_ir;
  }
  c->nlev_bad |= bad;
  free(te);
}

/* colrat(a+1,b+1) of cell q (the (ix,jx,kx,6,6) array: plane a + 6*b). */
#define NL_CR(c, q, a, b) ((c)->colrat[(q) + (size_t)((a) + 6 * (b)) * (c)->nc])

/* derivative (Scheme_rot.f90:692-736) of plane v along dir (1 or 2): order 4 (s_order 4's
 * five-point form) or 1 (s_order 1's two-point form); 0 leaves der at zero.  Cells the
 * stencil does not reach are zero here (the reference leaves them unset, and its s_order 2
 * sets no cell at all). */
static void nl_derivative(const orc_ctx *c, const double *v, double *der, int dir) {
  int ix = c->ix, jx = c->jx, order = c->nlev_deriv;
  memset(der, 0, sizeof(double) * c->nc);
  if (order == 0) return;
  int w = order == 4 ? 2 : 1;
  for (int j = 0; j < jx; ++j)
    for (int i = 0; i < ix; ++i) {
      size_t q = AT(c, i, j, 0);
      if (dir == 1) {
        if (i < w || i >= ix - w) continue;
        if (order == 4)
          der[q] = (-v[q + 2] + 8.0 * v[q + 1] - 8.0 * v[q - 1] + v[q - 2]) / (12.0 * c->dx[i]);
        else
          der[q] = (v[q + 1] - v[q - 1]) / (2.0 * c->dx[i]);
      } else {
        if (j < w || j >= jx - w) continue;
        size_t s = (size_t)ix;
        if (order == 4)
          der[q] = (-v[q + 2 * s] + 8.0 * v[q + s] - 8.0 * v[q - s] + v[q - 2 * s]) /
                   (12.0 * c->dy[j]);
        else
          der[q] = (v[q + s] - v[q - s]) / (2.0 * c->dy[j]);
      }
    }
}

/* The convective term of level ii (0-based) at every cell: d(Nexcite)/dx*vx_n (+ y). */
static void nl_conv(const orc_ctx *c, int ii, double *conv, double *tmp) {
  size_t nc = c->nc;
  const double *Uh = c->U_h, *v = c->nex + ii * nc;
  nl_derivative(c, v, tmp, 1);
  for (size_t q = 0; q < nc; ++q) conv[q] = tmp[q] * Uh[q + nc] / Uh[q];
  if (c->p.ndim > 1) {
    nl_derivative(c, v, tmp, 2);
    for (size_t q = 0; q < nc; ++q) conv[q] = conv[q] + tmp[q] * Uh[q + 2 * nc] / Uh[q];
  }
}

/* hydrogen_excitation_timestep (Scheme_rot.f90:1002-1049) reduced by cfl_pip_ir_nexcite
 * (:329-335): max over every cell and levels 1-5 of dNexcite/dt. */
static double nl_dneut_max(orc_ctx *c) {
  size_t nc = c->nc;
  double gref = c->gm_rec_ref, tir = c->p.t_ir;
  double *conv = malloc(sizeof(double) * nc * 5), *tmp = malloc(sizeof(double) * nc);
  for (int ii = 0; ii < 5; ++ii) nl_conv(c, ii, conv + ii * nc, tmp);
  double mx = -INFINITY;
  for (size_t q = 0; q < nc; ++q) {
    double nx[6];
    for (int k = 0; k < 6; ++k) nx[k] = c->nex[q + k * nc];
    for (int ii = 0; ii < 5; ++ii) {
      double d = 0.0;
      for (int jj = 0; jj < 6; ++jj)
        d = d + nx[jj] * NL_CR(c, q, jj, ii) / gref * tir - nx[ii] * NL_CR(c, q, ii, jj) / gref * tir;
      mx = fmx(mx, d - conv[q + ii * nc]);
    }
  }
  free(conv);
  free(tmp);
  return mx;
}

/* boundary of one scalar plane (bnd_energy, Boundary_rot.f90:127-162): the type mapping of
 * MHDbnd, sign +1 (the energy's entry of sym_mhd). */
static void nl_bnd_plane(orc_ctx *c, double *v) {
  static const int one[1] = {1};
  for (int f = 0; f < 2 * c->p.ndim; ++f)
    if (c->neighbor[f] == -1) boundary_control(c, v, 1, f / 2 + 1, f % 2, one, bnd_type(c->p.flag_bnd[f]));
}

/* hydrogen_excitation_update (PIP_rot.f90:1026-1159) over dt, after a stage's update of U
 * (Solver_rot.f90:218-220): the ion population's sum first, then the neutral levels' sums
 * over the ion and over the other levels, minus the convection by the neutral velocity;
 * the 1e-16 floor, the ground level absorbing the difference to rho_n, Nexcite(6) = rho_i,
 * and bnd_energy on every plane. */
static void hydrogen_excitation_update(orc_ctx *c, double dt) {
  size_t nc = c->nc;
  double gref = c->gm_rec_ref, tir = c->p.t_ir;
  double *conv = malloc(sizeof(double) * nc * 5), *tmp = malloc(sizeof(double) * nc);
  for (int ii = 0; ii < 5; ++ii) nl_conv(c, ii, conv + ii * nc, tmp);
  double *N = c->nex;
  const double *Uh = c->U_h, *Um = c->U_m;
  for (size_t q = 0; q < nc; ++q) {
    double nx[6], d[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < 6; ++k) nx[k] = N[q + k * nc];
    for (int jj = 0; jj < 5; ++jj)
      d[5] = d[5] + nx[jj] * NL_CR(c, q, jj, 5) / gref * tir - nx[5] * NL_CR(c, q, 5, jj) / gref * tir;
    for (int ii = 0; ii < 5; ++ii)
      d[ii] = d[ii] + nx[5] * NL_CR(c, q, 5, ii) / gref * tir - nx[ii] * NL_CR(c, q, ii, 5) / gref * tir;
    for (int ii = 0; ii < 5; ++ii)
      for (int jj = 0; jj < 5; ++jj)
        d[ii] = d[ii] + nx[jj] * NL_CR(c, q, jj, ii) / gref * tir - nx[ii] * NL_CR(c, q, ii, jj) / gref * tir;
    for (int ii = 0; ii < 5; ++ii) {
      double v = nx[ii] + dt * (d[ii] - conv[q + ii * nc]);
      nx[ii] = v > NL_FLOOR ? v : NL_FLOOR;
    }
    double tot = nx[0] + nx[1] + nx[2] + nx[3] + nx[4] - Uh[q];
    nx[0] = nx[0] - tot;
    nx[5] = Um[q];
    for (int k = 0; k < 6; ++k) N[q + k * nc] = nx[k];
  }
  for (int k = 0; k < 6; ++k) nl_bnd_plane(c, N + k * nc);
  free(conv);
  free(tmp);
}

int orc_set_nlevel(orc_ctx *c, int deriv, double n0fac, double f_p_ini, double f_p_p_ini,
                   const double *table, long nrows) {
  if (c->p.flag_ir != PIP_IR_NLEVEL || nrows < 3 || (deriv != 0 && deriv != 1 && deriv != 4))
    return PIP_ERR_PARAM;
  c->nlev_deriv = deriv;
  c->n0fac = n0fac;
  c->f_p_ini = f_p_ini;
  c->f_p_p_ini = f_p_p_ini;
  free(c->etab);
  c->etab = malloc(sizeof(double) * 4 * nrows);
  memcpy(c->etab, table, sizeof(double) * 4 * nrows);
  c->netab = nrows;
  nl_constants(c);
  if (!c->nex) c->nex = calloc(c->nc * 6, sizeof(double));
  if (!c->colrat) c->colrat = calloc(c->nc * 36, sizeof(double));
  if (!c->ion_pot) c->ion_pot = calloc(c->nc, sizeof(double));
  c->nlev_init = 0;
  c->init_done = 0;
  return 0;
}

void orc_set_nexcite(orc_ctx *c, const double *nex) {
  memcpy(c->nex, nex, sizeof(double) * c->nc * 6);
}
void orc_get_nexcite(const orc_ctx *c, double *nex) {
  memcpy(nex, c->nex, sizeof(double) * c->nc * 6);
}
void orc_get_colrat(const orc_ctx *c, double *colrat) {
  memcpy(colrat, c->colrat, sizeof(double) * c->nc * 36);
}
void orc_get_ion_pot(const orc_ctx *c, double *ion_pot) {
  memcpy(ion_pot, c->ion_pot, sizeof(double) * c->nc);
}
double orc_gm_rec_ref(const orc_ctx *c) { return c->gm_rec_ref; }
int orc_nlevel_status(const orc_ctx *c) { return c->nlev_bad; }

/* set_IR types 1, 2 and 3 (PIP_rot.f90:134-228): get_Te_HD and get_Te_MHD rewrite both
 * energies, then the rates from the ion temperature Te_p and density.  Type 1 (the Jeffery
 * formulation, :135-149) from T_norm and n_norm; types 2 and 3 the Popescu et al. 2019 rates
 * with the electron temperature Te_0 = T_norm/1.1604e4 eV.  The single-precision literals of
 * the Fortran (2.7, 5.6e-16, 1.1604e4, 2.6e-19, 2.91e-14, 1.0e6) are rounded to float first,
 * as there. */
static void set_ir_law(orc_ctx *c) {
  const pip_params *p = &c->p;
  size_t nc = c->nc;
  if (p->flag_ir == PIP_IR_NLEVEL) {
    set_ir_nlevel(c);
    return;
  }
  if (p->flag_ir == PIP_IR_JEFFERY) {
    double T0 = p->t_norm, n0 = p->n_norm;
    double factor = exp(-13.2 / (T0 / 11605.0));
    double factor2 = (double)2.7f * pow(13.2 * 11605.0, -2.0) * pow(T0, 1.0 / 2.0) * n0;
    double factor3 = (double)5.6e-16f * pow(13.2 * 11605.0, -2.0) * pow(T0, -1.0) * pow(n0, 2.0);
    double rec_fac = factor2 / factor3, ion_fac = factor3 / p->t_ir;
    const double *Um1 = c->U_m;
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < nc; ++q) {
      double te_p, te_n;
      get_te_cell(c, q, &te_p, &te_n);
      double ro = Um1[q];
      c->gm_rec[q] = pow(te_p, -0.5) * (ro * ro) * rec_fac * ion_fac;
      c->gm_ion[q] = pow(te_p, 0.5) * ro * pow(factor, 1.0 / te_p) * ion_fac;
    }
    return;
  }
  double t_ir = p->t_ir, n6 = p->n_norm * (double)1.0e6f;
  double Te_0 = p->t_norm / (double)1.1604e4f;
  double c26 = (double)2.6e-19f, c291 = (double)2.91e-14f;
  int law = p->flag_ir;
  double rec2 = c26 * n6 / sqrt(Te_0) * t_ir;            /* type 2 rec_fac */
  double rec3 = c26 * n6 / sqrt(Te_0);                   /* type 3 rec_fac */
  double ioneq = (c26 / sqrt(Te_0)) /
                 (c291 / (0.232 + 13.6 / Te_0) * pow(13.6 / Te_0, 0.39) * exp(-13.6 / Te_0));
  double f_n = ioneq / (ioneq + 1.0), f_p = 1.0 - f_n, f_p_p = 2.0 * f_p / (f_n + 2.0 * f_p);
  double tfac = (p->flag_col % 2 == 1) ? 0.5 * f_p_p / f_p
                                       : p->beta / 2.0 * f_p_p * 5.0 / 6.0 / f_p;
  const double *Um = c->U_m;
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < nc; ++q) {
    double te_p, te_n;
    get_te_cell(c, q, &te_p, &te_n);
    double ro = Um[q];
    if (law == PIP_IR_POPESCU) {
      double a = 13.6 / Te_0 / te_p;
      c->gm_rec[q] = ro / sqrt(te_p) * rec2;
      c->gm_ion[q] = (n6 * ro) * c291 * exp(-13.6 / Te_0 / te_p) * pow(a, 0.39) / (0.232 + a) * t_ir;
    } else {
      double b = 13.6 / Te_0 / te_p * tfac;
      c->gm_rec[q] = ro / sqrt(te_p) * t_ir / f_p * sqrt(tfac);
      double g = c291 * n6 * ro * exp(-13.6 / Te_0 / te_p * tfac) * pow(b, 0.39);
      c->gm_ion[q] = g / (0.232 + b) / rec3 / f_p * t_ir;
    }
  }
}

static int ir_per_stage(const orc_ctx *c) {
  return c->p.flag_ir == PIP_IR_POPESCU || c->p.flag_ir == PIP_IR_POPESCU_EQ ||
         c->p.flag_ir == PIP_IR_NLEVEL;
}

/* set_IR types 1-3: called by the time loop before each cfl and at the prologue */
static int ir_loop(const orc_ctx *c) {
  return ir_per_stage(c) || c->p.flag_ir == PIP_IR_JEFFERY;
}

/* set_coefficients(U_h,U_m,0) of the prologue (Initial_rot.f90:140), on the state as it
 * stands, before the first call that reads the state: set_collisional (alpha_c per cell)
 * and set_IR (the Popescu laws), each with get_Te's energy rewrite. */
static void ensure_coefficients(orc_ctx *c) {
  if (c->init_done) return;
  if (c->resi == 2) set_resistivity_anomalous(c);
  if (c->col_type >= 1) set_collisional(c);
  if (ir_loop(c)) set_ir_law(c);
  c->init_done = 1;
}

void orc_ir_rates(const orc_ctx *c, double *gm_ion, double *gm_rec) {
  memcpy(gm_ion, c->gm_ion, sizeof(double) * c->nc);
  memcpy(gm_rec, c->gm_rec, sizeof(double) * c->nc);
}

void orc_coefficients(orc_ctx *c) {
  if (c->resi == 2) set_resistivity_anomalous(c);
  if (c->col_type >= 1) set_collisional(c);
  if (ir_loop(c)) set_ir_law(c);
  c->init_done = 1;
}

int orc_alpha_c(orc_ctx *c, double *ac) {
  size_t nc = c->nc;
  ensure_coefficients(c);
  for (size_t q = 0; q < nc; ++q) ac[q] = c->col_type >= 1 ? c->ac[q] : c->p.col;
  return 0;
}

/* source_PIP, PIP_rot.f90:1309-1429 (explicit and exponential collision forms plus the
 * IR block with flag_IR_type 1 or 2, and 0 with set_IR type 4).  out_h/out_m receive S (explicit form) or the U0
 * increments of the exponential form, plus the IR rates in S. */
static void source_pip(orc_ctx *c, double *U_h0, double *U_m0, double dt_coll, double *S_h,
                       double *S_m) {
  size_t nc = c->nc;
  double gm = c->p.gm;
  const double *acf = c->col_type >= 1 ? c->ac : NULL;
  double *w = malloc(sizeof(double) * nc * 13);
  double *nde = w, *nvx = w + nc, *nvy = w + 2 * nc, *nvz = w + 3 * nc, *npr = w + 4 * nc;
  double *de = w + 5 * nc, *vx = w + 6 * nc, *vy = w + 7 * nc, *vz = w + 8 * nc, *pr = w + 9 * nc;
  cq2pv_hd(c, c->U_h, nde, nvx, nvy, nvz, npr);
  cq2pv_mhd(c, c->U_m, de, vx, vy, vz, pr, NULL, NULL, NULL);
  double *U_h = c->U_h, *U_m = c->U_m;
  int imp = c->p.flag_pip_imp == 1;
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < nc; ++q) {
    double ac = acf ? acf[q] : c->p.col;
    double te = pr[q] / de[q] * gm * MU_P;
    double nte = npr[q] / nde[q] * gm * MU_N;
    double ds[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (imp) {
      double temp = dt_coll * (U_h[q] + U_m[q]);
      double e = (1.0 - exp(-ac * temp));
      ds[1] = (U_m[q] * U_h[q + nc] - U_h[q] * U_m[q + nc]) * e / temp;
      ds[2] = (U_m[q] * U_h[q + 2 * nc] - U_h[q] * U_m[q + 2 * nc]) * e / temp;
      ds[3] = (U_m[q] * U_h[q + 3 * nc] - U_h[q] * U_m[q + 3 * nc]) * e / temp;
      double lambda = ac * (nde[q] + de[q]);
      double kap = 3.0 * (gm - 1.0) * ac * (MU_P * nde[q] + MU_N * de[q]);
      double dvx = nvx[q] - vx[q], dvy = nvy[q] - vy[q], dvz = nvz[q] - vz[q];
      /* (nvz-vz)*nvz in the ion term is as written in PIP_rot.f90:1348 */
      double B = -(1.0 / 3.0 * gm * kap / ((nde[q] + de[q]) * (kap - lambda)) *
                   (de[q] * (dvx * vx[q] + dvy * vy[q] + dvz * nvz[q]) +
                    nde[q] * (dvx * nvx[q] + dvy * nvy[q] + dvz * nvz[q])));
      double D = -(gm / 6.0 * kap * (de[q] - nde[q]) / ((de[q] + nde[q]) * (kap - 2.0 * lambda)) *
                   (dvx * dvx + dvy * dvy + dvz * dvz));
      ds[4] = -((3.0 / gm) * ac * de[q] * nde[q] / kap *
                (+(exp(-kap * dt_coll) - 1.0) * (nte - te) - (B + D) * exp(-kap * dt_coll) +
                 B * exp(-lambda * dt_coll) + D * exp(-2.0 * lambda * dt_coll)) /
                dt_coll);
      for (int n = 0; n < 5; ++n) {
        U_h0[q + n * nc] = U_h0[q + n * nc] - dt_coll * ds[n];
        U_m0[q + n * nc] = U_m0[q + n * nc] + dt_coll * ds[n];
      }
    } else {
      ds[1] = ac * (U_m[q] * U_h[q + nc] - U_h[q] * U_m[q + nc]);
      ds[2] = ac * (U_m[q] * U_h[q + 2 * nc] - U_h[q] * U_m[q + 2 * nc]);
      ds[3] = ac * (U_m[q] * U_h[q + 3 * nc] - U_h[q] * U_m[q + 3 * nc]);
      ds[4] = ac * nde[q] * de[q] *
              (0.5 * ((nvx[q] * nvx[q] - vx[q] * vx[q]) + (nvy[q] * nvy[q] - vy[q] * vy[q]) +
                      (nvz[q] * nvz[q] - vz[q] * vz[q])) +
               3.0 / gm / 2.0 * (nte - te));
      for (int n = 0; n < 5; ++n) {
        S_h[q + n * nc] = S_h[q + n * nc] - ds[n];
        S_m[q + n * nc] = S_m[q + n * nc] + ds[n];
      }
    }
    if (c->p.flag_ir != PIP_IR_NONE) {
      double gr = c->gm_rec[q], gi = c->gm_ion[q];
      ds[0] = gr * de[q] - gi * nde[q];
      ds[1] = gr * de[q] * vx[q] - gi * nde[q] * nvx[q];
      ds[2] = gr * de[q] * vy[q] - gi * nde[q] * nvy[q];
      ds[3] = gr * de[q] * vz[q] - gi * nde[q] * nvz[q];
      double kin = 0.5 * (gr * de[q] * (vx[q] * vx[q] + vy[q] * vy[q] + vz[q] * vz[q]) -
                          gi * nde[q] * (nvx[q] * nvx[q] + nvy[q] * nvy[q] + nvz[q] * nvz[q]));
      if (c->p.flag_ir_type != 2)
        ds[4] = kin - gi * npr[q] / (gm - 1.0) + 0.5 * gr * pr[q] / (gm - 1.0);
      else
        ds[4] = kin - gi * npr[q] / (gm - 1.0) + gr * pr[q] / (gm - 1.0);
      for (int n = 0; n < 5; ++n) {
        S_h[q + n * nc] = S_h[q + n * nc] + ds[n];
        S_m[q + n * nc] = S_m[q + n * nc] - ds[n];
      }
      if (c->p.flag_ir_type == 0) {
        /* the new formulation's ionisation potential (IRgetionpot for type 4; arb_heat 0) */
        double nx[6], cr[36];
        for (int k = 0; k < 6; ++k) nx[k] = c->nex[q + k * nc];
        for (int k = 0; k < 36; ++k) cr[(k % 6) * 6 + k / 6] = c->colrat[q + k * nc];
        c->ion_pot[q] = nl_ionpot(c, cr, nx);
        S_m[q + 4 * nc] = S_m[q + 4 * nc] - c->ion_pot[q] + 0.0;
      }
    }
  }
  free(w);
}

void orc_source(orc_ctx *c, double dt_coll, double *S_h, double *S_m) {
  size_t nc = c->nc;
  ensure_coefficients(c);
  memset(S_h, 0, sizeof(double) * nc * c->nh);
  memset(S_m, 0, sizeof(double) * nc * c->nm);
  /* the Popescu rates of the state as given (set_IR before set_source) */
  if (ir_per_stage(c)) set_ir_law(c);
  if (c->p.flag_pip_imp == 1) {
    /* report the U0 increments: run the form on zero U0 copies */
    source_pip(c, S_h, S_m, dt_coll, S_h, S_m);
  } else {
    source_pip(c, NULL, NULL, dt_coll, S_h, S_m);
  }
}

/* ---------------------------------------------------------------- CFL */

/* cfl, Scheme_rot.f90:183-213 with cfl_mhd :245-289, cfl_hd :215-243, cfl_pn_col :305-313
 * and cfl_pip_ir :315-327 (flag_IR_type 1/2 branch). */
void orc_cfl(orc_ctx *c, double *dt_out, double *cmax_out) {
  const pip_params *p = &c->p;
  size_t nc = c->nc;
  double gm = p->gm, safety = p->safety, ac = p->col;
  ensure_coefficients(c);
  const double *acf = c->col_type >= 1 ? c->ac : NULL;
  double *w = malloc(sizeof(double) * nc * 8);
  double *de = w, *vx = w + nc, *vy = w + 2 * nc, *vz = w + 3 * nc, *pr = w + 4 * nc;
  double *bx = w + 5 * nc, *by = w + 6 * nc, *bz = w + 7 * nc;
  int m0 = p->margin[0], m1 = p->margin[1], m2 = p->margin[2];

  /* set_IR of the time loop before each cfl (main.f90:32-34,44-46), set_IR types 1-3 */
  if (ir_loop(c)) set_ir_law(c);
  /* cfl_mhd */
  cq2pv_mhd(c, c->U_m, de, vx, vy, vz, pr, bx, by, bz);
  /* set_IR for the rates the following run_solver uses: from the rewritten ion state */
  if (p->flag_ir == PIP_IR_POWERLAW) set_ir_rates(c);
  double dt_min = 10.0;
#pragma omp parallel for collapse(2) reduction(min : dt_min) schedule(static)
  for (int k = m2; k < c->kx - m2; ++k)
    for (int j = m1; j < c->jx - m1; ++j)
      for (int i = m0; i < c->ix - m0; ++i) {
        size_t q = AT(c, i, j, k);
        double gmin = fmn(fmn(c->dx[i], c->dy[j]), c->dz[k]);
        double cs2 = gm * pr[q] / fmx(de[q], TINY);
        double valf2 = (bx[q] * bx[q] + by[q] * by[q] + bz[q] * bz[q]) / fmx(de[q], TINY);
        double vabs = sqrt(vx[q] * vx[q] + vy[q] * vy[q] + vz[q] * vz[q]);
        dt_min = fmn(dt_min, safety * gmin / (vabs + sqrt(cs2 + valf2)));
      }
  double dttemp = dt_min;

  /* cfl_hd (flag_pip=1: starts from the MHD value) */
  cq2pv_hd(c, c->U_h, de, vx, vy, vz, pr);
  dt_min = dttemp;
#pragma omp parallel for collapse(2) reduction(min : dt_min) schedule(static)
  for (int k = m2; k < c->kx - m2; ++k)
    for (int j = m1; j < c->jx - m1; ++j)
      for (int i = m0; i < c->ix - m0; ++i) {
        size_t q = AT(c, i, j, k);
        double gmin = fmn(fmn(c->dx[i], c->dy[j]), c->dz[k]);
        double cs = sqrt(gm * pr[q] / de[q]);
        double vabs = sqrt(fmx(vx[q] * vx[q] + vy[q] * vy[q] + vz[q] * vz[q], TINY));
        dt_min = fmn(dt_min, safety * gmin / (vabs + cs));
      }
  dttemp = dt_min;

  /* cfl_pn_col: maxima over all cells, ghosts included */
  double mm = -INFINITY, mh = -INFINITY;
#pragma omp parallel for reduction(max : mm, mh) schedule(static)
  for (size_t q = 0; q < nc; ++q) {
    double a = acf ? acf[q] : ac;
    mm = fmx(mm, c->U_m[q] * a);
    mh = fmx(mh, c->U_h[q] * a);
  }
  if (p->flag_pip_imp == 1) dttemp = fmn(dttemp, p->pip_imp_factor / fmx(mm, mh));
  else dttemp = fmn(dttemp, fmn(safety, 0.3) / fmx(mm, mh));

  /* cfl_pip_ir */
  if (p->flag_ir != PIP_IR_NONE) {
    double gr = -INFINITY, gi = -INFINITY;
#pragma omp parallel for reduction(max : gr, gi) schedule(static)
    for (size_t q = 0; q < nc; ++q) {
      gr = fmx(gr, c->gm_rec[q]);
      gi = fmx(gi, c->gm_ion[q]);
    }
    dttemp = fmn(dttemp, fmn(safety, 0.1) / fmx(fmx(gr, gi), 1.0e-5));
    if (p->flag_ir_type == 0) {
      /* get_Pr_MHD (Scheme_rot.f90:112-128, rewriting the ion energy once more), then
       * ion_pot of the last source_PIP (or of the prologue) over the internal energy */
      double ipm = -INFINITY;
      double *Um = c->U_m;
      for (size_t q = 0; q < nc; ++q) {
        double m1 = Um[q], m2 = Um[q + nc], m3 = Um[q + 2 * nc], m4 = Um[q + 3 * nc];
        double m6 = Um[q + 5 * nc], m7 = Um[q + 6 * nc], m8 = Um[q + 7 * nc];
        double prm = (gm - 1.0) * (Um[q + 4 * nc] -
                                   0.5 * ((m2 * m2 + m3 * m3 + m4 * m4) / m1 + m6 * m6 + m7 * m7 + m8 * m8));
        prm = fmx(prm, p->pr_lim);
        Um[q + 4 * nc] = prm / (gm - 1.0) + 0.5 * ((m2 * m2 + m3 * m3 + m4 * m4) / m1 + m6 * m6 +
                                                   m7 * m7 + m8 * m8);
        ipm = fmx(ipm, c->ion_pot[q] / (prm / (gm - 1.0)));
      }
      dttemp = fmn(dttemp, safety / fmx(ipm, 1.0e-5));
    }
    if (p->flag_ir == PIP_IR_NLEVEL)
      dttemp = fmn(dttemp, fmn(safety, 0.01) / fmx(nl_dneut_max(c), 1.0e-5));
  }

  /* cfl_resi (Scheme_rot.f90:291-302) */
  if (c->resi) dttemp = cfl_resi(c, dttemp);

  /* cmax for Dedner cleaning */
  double cmax = c->cmax;
  if (p->flag_divb >= 1) {
    double g = INFINITY;
    for (int i = 0; i < c->ix; ++i) g = fmn(g, c->dx[i]);
    double gy = INFINITY, gz = INFINITY;
    for (int j = 0; j < c->jx; ++j) gy = fmn(gy, c->dy[j]);
    for (int k = 0; k < c->kx; ++k) gz = fmn(gz, c->dz[k]);
    g = fmn(fmn(g, gy), gz);
    cmax = safety * g / dttemp;
  }
  free(w);
  if (dt_out) *dt_out = dttemp;
  if (cmax_out) *cmax_out = cmax;
}

/* cfl_resi (Scheme_rot.f90:291-302): dt lowered to safety*gmin**2/max(eta,1e-8) over the
 * interior cells.  It writes the global dt, whatever variable the enclosing cfl call
 * fills: in the time loop's first cfl that is the step's dt, in the second (after
 * run_solver) the dt that `time` then advances by (main.f90:47,58). */
static double cfl_resi(orc_ctx *c, double dt) {
  const pip_params *p = &c->p;
  const int m0 = p->margin[0], m1 = p->margin[1], m2 = p->margin[2];
  const double safety = p->safety, etmin = 1.0e-8;
  double dr = dt;
#pragma omp parallel for collapse(2) reduction(min : dr) schedule(static)
  for (int k = m2; k < c->kx - m2; ++k)
    for (int j = m1; j < c->jx - m1; ++j)
      for (int i = m0; i < c->ix - m0; ++i) {
        double gmin = fmn(fmn(c->dx[i], c->dy[j]), c->dz[k]);
        dr = fmn(dr, safety * (gmin * gmin) / fmx(c->eta[AT(c, i, j, k)], etmin));
      }
  return dr;
}

/* ---------------------------------------------------------------- integration */

/* add_flux_rk HLL branch, Solver_rot.f90:383-405. */
static void add_flux_rk(orc_ctx *c, const double *F, const double *U0, double *U, int nvar,
                        double dt, int dir) {
  size_t nc = c->nc;
  int ix = c->ix, jx = c->jx, kx = c->kx;
  if (dir == 1) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int n = 0; n < nvar; ++n)
      for (int k = 0; k < kx; ++k)
        for (int j = 0; j < jx; ++j)
          for (int i = 1; i < ix; ++i) {
            size_t q = AT(c, i, j, k) + n * nc;
            U[q] = U0[q] - (dt / c->dx[i]) * (F[q] - F[q - 1]);
          }
  } else if (dir == 2) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int n = 0; n < nvar; ++n)
      for (int k = 0; k < kx; ++k)
        for (int j = 1; j < jx; ++j)
          for (int i = 0; i < ix; ++i) {
            size_t q = AT(c, i, j, k) + n * nc;
            U[q] = U[q] - (dt / c->dy[j]) * (F[q] - F[q - ix]);
          }
  }
}

/* ---------------------------------------------------------------- implicit conduction */

/* Stencil of the 9-point matrix (initialize_HC, HC_rot.f90:41-46, hc_split=2): entries
 * 0..8 couple cell (i,j) with (i,j), (i-1,j), (i+1,j), (i,j-1), (i,j+1), (i-1,j-1),
 * (i+1,j-1), (i-1,j+1), (i+1,j+1). */
#define HC_EPSI 1.0e-5               /* HC_rot.f90:17 */

/* matrix(i,j,:) . v over the 9-point stencil, summed left to right as the Fortran does. */
static double hc_apply(const orc_ctx *c, const double *mat, const double *v, size_t q) {
  const size_t nc = c->nc;
  const long ix = c->ix;
  return mat[q] * v[q] + mat[q + nc] * v[q - 1] + mat[q + 2 * nc] * v[q + 1] +
         mat[q + 3 * nc] * v[q - ix] + mat[q + 4 * nc] * v[q + ix] +
         mat[q + 5 * nc] * v[q - 1 - ix] + mat[q + 6 * nc] * v[q + 1 - ix] +
         mat[q + 7 * nc] * v[q - 1 + ix] + mat[q + 8 * nc] * v[q + 1 + ix];
}

/* set_matrix_source_MHD2D9 (HC_rot.f90:643-739) for the interior cells (dxc = dx and
 * dyc = dy for s_order = 2, Model_rot.f90:430-431), then set_matrix_boundary
 * (HC_rot.f90:468-529) on the sides whose neighbour is -1: the stencil entries outside the
 * domain are folded onto the boundary row (x-, x+, y-, y+ in that order).  With one rank
 * per direction every neighbour is -1 (set_mpi_neighbor, MPI_rot.f90:123). */
static void hc_matrix(const orc_ctx *c, const double *ro, const double *te, const double *bx,
                      const double *by, const double *bz, double dt, double *mat) {
  const pip_params *p = &c->p;
  const size_t nc = c->nc;
  const int ix = c->ix, jx = c->jx;
  const int is = p->margin[0], ie = ix - p->margin[0] - 1;
  const int js = p->margin[1], je = jx - p->margin[1] - 1;
  const double gm = p->gm, kapper = p->kapper;
  for (int j = js; j <= je; ++j)
    for (int i = is; i <= ie; ++i) {
      const size_t q = (size_t)j * ix + i;
      const double eta = kapper * dt * (gm - 1.0) / ro[q] * gm;
      const double bxl = (bx[q - 1] + bx[q]) / 2.0, bxr = (bx[q + 1] + bx[q]) / 2.0;
      const double bxd = (bx[q - ix] + bx[q]) / 2.0, bxu = (bx[q + ix] + bx[q]) / 2.0;
      const double byl = (by[q - 1] + by[q]) / 2.0, byr = (by[q + 1] + by[q]) / 2.0;
      const double byd = (by[q - ix] + by[q]) / 2.0, byu = (by[q + ix] + by[q]) / 2.0;
      const double bzl = (bz[q - 1] + bz[q]) / 2.0, bzr = (bz[q + 1] + bz[q]) / 2.0;
      const double bzd = (bz[q - ix] + bz[q]) / 2.0, bzu = (bz[q + ix] + bz[q]) / 2.0;
      const double nxl = bxl / (fmx(sqrt(bxl * bxl + byl * byl + bzl * bzl), HC_EPSI));
      const double nxr = bxr / (fmx(sqrt(bxr * bxr + byr * byr + bzr * bzr), HC_EPSI));
      const double nxd = bxd / (fmx(sqrt(bxd * bxd + byd * byd + bzd * bzd), HC_EPSI));
      const double nxu = bxu / (fmx(sqrt(bxu * bxu + byu * byu + bzu * bzu), HC_EPSI));
      const double nyl = byl / (fmx(sqrt(bxl * bxl + byl * byl + bzl * bzl), HC_EPSI));
      const double nyr = byr / (fmx(sqrt(bxr * bxr + byr * byr + bzr * bzr), HC_EPSI));
      const double nyd = byd / (fmx(sqrt(bxd * bxd + byd * byd + bzd * bzd), HC_EPSI));
      const double nyu = byu / (fmx(sqrt(bxu * bxu + byu * byu + bzu * bzu), HC_EPSI));
      const double te_xm = 0.5 * (te[q] + te[q - 1]), te_xp = 0.5 * (te[q] + te[q + 1]);
      const double te_ym = 0.5 * (te[q] + te[q - ix]), te_yp = 0.5 * (te[q] + te[q + ix]);
      const double te_xm25 = te_xm * te_xm * sqrt(te_xm), te_xp25 = te_xp * te_xp * sqrt(te_xp);
      const double te_ym25 = te_ym * te_ym * sqrt(te_ym), te_yp25 = te_yp * te_yp * sqrt(te_yp);
      const double dxc = c->dx[i], dyc = c->dy[j];
      const double bxxl = -(eta * te_xm25 * nxl * nxl / dxc / c->dx[i - 1]);
      const double bxxr = -(eta * te_xp25 * nxr * nxr / dxc / c->dx[i]);
      const double byyd = -(eta * te_ym25 * nyd * nyd / dyc / c->dy[j - 1]);
      const double byyu = -(eta * te_yp25 * nyu * nyu / dyc / c->dy[j]);
      const double bxyl = -(eta / 4.0 / dxc / dyc * nxl * nyl * te_xm25);
      const double bxyr = -(eta / 4.0 / dxc / dyc * nxr * nyr * te_xp25);
      const double byxd = -(eta / 4.0 / dxc / dyc * nyd * nxd * te_ym25);
      const double byxu = -(eta / 4.0 / dxc / dyc * nyu * nxu * te_yp25);
      double *m = mat + q;
      m[nc] = bxxl - (byxu - byxd);
      m[2 * nc] = bxxr + (byxu - byxd);
      m[3 * nc] = byyd - (bxyr - bxyl);
      m[4 * nc] = byyu + (bxyr - bxyl);
      m[5 * nc] = bxyl + byxd;
      m[6 * nc] = -(bxyr + byxd);
      m[7 * nc] = -(bxyl + byxu);
      m[8 * nc] = bxyr + byxu;
      m[0] = 1.0 - (m[nc] + m[2 * nc] + m[3 * nc] + m[4 * nc]);
    }
  /* set_matrix_boundary, hc_split = 2 (entries 1..9 of the Fortran are 0..8 here) */
#define M(n, qq) mat[(size_t)(n) * nc + (qq)]
  for (int j = js; j <= je && c->neighbor[0] == -1; ++j) {       /* x-minus */
    const size_t q = (size_t)j * ix + is;
    M(0, q) = M(1, q) + M(0, q); M(1, q) = 0.0;
    M(3, q) = M(3, q) + M(5, q); M(5, q) = 0.0;
    M(4, q) = M(4, q) + M(7, q); M(7, q) = 0.0;
  }
  for (int j = js; j <= je && c->neighbor[1] == -1; ++j) {       /* x-plus */
    const size_t q = (size_t)j * ix + ie;
    M(0, q) = M(2, q) + M(0, q); M(2, q) = 0.0;
    M(3, q) = M(3, q) + M(6, q); M(6, q) = 0.0;
    M(4, q) = M(4, q) + M(8, q); M(8, q) = 0.0;
  }
  for (int i = is; i <= ie && c->neighbor[2] == -1; ++i) {       /* y-minus */
    const size_t q = (size_t)js * ix + i;
    M(0, q) = M(3, q) + M(0, q); M(3, q) = 0.0;
    M(1, q) = M(5, q) + M(1, q); M(5, q) = 0.0;
    M(2, q) = M(6, q) + M(2, q); M(6, q) = 0.0;
  }
  for (int i = is; i <= ie && c->neighbor[3] == -1; ++i) {       /* y-plus */
    const size_t q = (size_t)je * ix + i;
    M(0, q) = M(4, q) + M(0, q); M(4, q) = 0.0;
    M(1, q) = M(1, q) + M(7, q); M(7, q) = 0.0;
    M(2, q) = M(2, q) + M(8, q); M(8, q) = 0.0;
  }
#undef M
}

/* BiCGstab (HC_rot.f90:187-299, hc_split = 2): the residual is recomputed from te every
 * iteration; stops when sqrt(sum r^2 / sum b^2) <= hc_error or after hc_max+1 iterations.
 * Sums run in the Fortran array order.  Entries of the Krylov vectors outside the interior
 * are zero (the folded matrix multiplies them by exact zeros). */
static int hc_bicgstab(const orc_ctx *c, const double *mat, double *te, const double *src,
                       int *count_out, double *relres_out) {
  const pip_params *p = &c->p;
  const size_t nc = c->nc;
  const int ix = c->ix, jx = c->jx;
  const int is = p->margin[0], ie = ix - p->margin[0] - 1;
  const int js = p->margin[1], je = jx - p->margin[1] - 1;
  double *r = calloc(nc, sizeof(double)), *r0 = calloc(nc, sizeof(double));
  double *pk = calloc(nc, sizeof(double)), *apk = calloc(nc, sizeof(double));
  double *tkp = calloc(nc, sizeof(double));
  double total_resi = 0.0, total_source = 0.0;
  for (int j = js; j <= je; ++j)
    for (int i = is; i <= ie; ++i) {
      const size_t q = (size_t)j * ix + i;
      double v = src[q];
      v = v - mat[q] * te[q];
      v = v - mat[q + nc] * te[q - 1];
      v = v - mat[q + 2 * nc] * te[q + 1];
      v = v - mat[q + 3 * nc] * te[q - ix];
      v = v - mat[q + 4 * nc] * te[q + ix];
      v = v - mat[q + 5 * nc] * te[q - 1 - ix];
      v = v - mat[q + 6 * nc] * te[q + 1 - ix];
      v = v - mat[q + 7 * nc] * te[q - 1 + ix];
      v = v - mat[q + 8 * nc] * te[q + 1 + ix];
      r[q] = v;
      total_resi += v * v;
      total_source += src[q] * src[q];
      r0[q] = v;
      pk[q] = v;
    }
  int count = 0;
  const double error = p->hc_error;
  while (sqrt(total_resi / total_source) > error && count <= p->hc_max) {
    double alphau = 0.0, alphad = 0.0;
    for (int j = js; j <= je; ++j)
      for (int i = is; i <= ie; ++i) {
        const size_t q = (size_t)j * ix + i;
        apk[q] = hc_apply(c, mat, pk, q);
        alphau = alphau + (r[q] * r0[q]);
        alphad = alphad + (r0[q] * apk[q]);
      }
    const double alpha = alphau / alphad;
    for (int j = js; j <= je; ++j)
      for (int i = is; i <= ie; ++i) {
        const size_t q = (size_t)j * ix + i;
        tkp[q] = r[q] - alpha * apk[q];
      }
    double omegau = 0.0, omegad = 0.0;
    for (int j = js; j <= je; ++j)
      for (int i = is; i <= ie; ++i) {
        const size_t q = (size_t)j * ix + i;
        const double atk = hc_apply(c, mat, tkp, q);
        omegau = omegau + tkp[q] * atk;
        omegad = omegad + atk * atk;
      }
    const double omega = omegau / omegad;
    for (int j = js; j <= je; ++j)
      for (int i = is; i <= ie; ++i) {
        const size_t q = (size_t)j * ix + i;
        te[q] = te[q] + alpha * pk[q] + omega * tkp[q];
      }
    double betau = 0.0;
    total_resi = 0.0;
    for (int j = js; j <= je; ++j)
      for (int i = is; i <= ie; ++i) {
        const size_t q = (size_t)j * ix + i;
        r[q] = src[q] - hc_apply(c, mat, te, q);
        betau = betau + r0[q] * r[q];
        total_resi = total_resi + r[q] * r[q];
      }
    const double beta = betau / alphau * alpha / omega;
    for (int j = js; j <= je; ++j)
      for (int i = is; i <= ie; ++i) {
        const size_t q = (size_t)j * ix + i;
        pk[q] = r[q] + beta * (pk[q] - omega * apk[q]);
      }
    count = count + 1;
  }
  const double relres = sqrt(total_resi / total_source);
  free(r); free(r0); free(pk); free(apk); free(tkp);
  if (count_out) *count_out = count;
  if (relres_out) *relres_out = relres;
  return relres <= error ? PIP_OK : PIP_ERR_ITER;
}

/* HC(U_m, nvar_m, 1) (HC_rot.f90:67-140) on one rank: cq2pv_mhd (rewriting U_m), te =
 * gm*(pr/ro), the matrix (source = te), BiCGstab, pr = (te*ro)/gm, pv2cq_mhd
 * (Scheme_rot.f90:43-79, flag_b_stg = 0).  Called by post_step (Solver_rot.f90:296-303)
 * when flag_heat = 1 with the implicit integration. */
int orc_conduction(orc_ctx *c, double dt, int *iters, double *relres) {
  const pip_params *p = &c->p;
  const size_t nc = c->nc;
  const double gm = p->gm;
  double *w = malloc(sizeof(double) * nc * 8);
  double *ro = w, *vx = w + nc, *vy = w + 2 * nc, *vz = w + 3 * nc, *pr = w + 4 * nc;
  double *bx = w + 5 * nc, *by = w + 6 * nc, *bz = w + 7 * nc;
  cq2pv_mhd(c, c->U_m, ro, vx, vy, vz, pr, bx, by, bz);
  double *te = malloc(sizeof(double) * nc), *src = malloc(sizeof(double) * nc);
  for (size_t q = 0; q < nc; ++q) {
    te[q] = gm * (pr[q] / ro[q]);
    src[q] = te[q];
  }
  double *mat = calloc(9 * nc, sizeof(double));
  hc_matrix(c, ro, te, bx, by, bz, dt, mat);
  const int st = hc_bicgstab(c, mat, te, src, iters, relres);
  double *U = c->U_m;
  for (size_t q = 0; q < nc; ++q) {
    pr[q] = (te[q] * ro[q]) / gm;
    U[q] = ro[q];
    U[q + nc] = ro[q] * vx[q];
    U[q + 2 * nc] = ro[q] * vy[q];
    U[q + 3 * nc] = ro[q] * vz[q];
    U[q + 4 * nc] = pr[q] / (gm - 1.0) + 0.5 * ro[q] * (vx[q] * vx[q] + vy[q] * vy[q] + vz[q] * vz[q]) +
                    0.5 * (bx[q] * bx[q] + by[q] * by[q] + bz[q] * bz[q]);
    U[q + 5 * nc] = bx[q];
    U[q + 6 * nc] = by[q];
    U[q + 7 * nc] = bz[q];
  }
  free(w); free(te); free(src); free(mat);
  return st;
}

/* BiCGstabMPI (HC_rot.f90:303-466, hc_split = 2) in the phases of pip_hcd_* for a block
 * whose faces with a neighbour (orc_set_neighbors) are not folded: begin (cq2pv, te, the
 * matrix, r = b - A te; sums (r,r), (b,b)), phase 0 (p = r), 1 (Ap = A p; sums (r,r0),
 * (r0,Ap)), 2 (t = r - alpha Ap, At; sums (t,At), (At,At)), 3 (x += alpha p + omega t), 4
 * (r = b - A x; sums (r0,r), (r,r)), 5 (p = r + beta (p - omega Ap)), end (the write-back of
 * orc_conduction).  The caller sums the scalars over the ranks and moves one row of r (after
 * begin and phase 4) and of Ap (after phase 1) across each exchanged face; t, x and p are
 * formed on every cell.  Interior sums run in the Fortran array order. */
enum { HCD_X = 0, HCD_B, HCD_R, HCD_R0, HCD_P, HCD_AP, HCD_T, HCD_NV };

static double *hcd_v(const orc_ctx *c, int k) { return c->hcd + (size_t)k * c->nc; }

int orc_hcd_begin(orc_ctx *c, double dt, double sums[2]) {
  const pip_params *p = &c->p;
  const size_t nc = c->nc;
  const double gm = p->gm;
  if (!c->hcd) c->hcd = calloc((HCD_NV + 9 + 8) * nc, sizeof(double));
  memset(c->hcd, 0, sizeof(double) * (HCD_NV + 9) * nc);
  double *mat = hcd_v(c, HCD_NV), *w = mat + 9 * nc;
  double *ro = w, *vx = w + nc, *vy = w + 2 * nc, *vz = w + 3 * nc, *pr = w + 4 * nc;
  double *bx = w + 5 * nc, *by = w + 6 * nc, *bz = w + 7 * nc;
  cq2pv_mhd(c, c->U_m, ro, vx, vy, vz, pr, bx, by, bz);
  double *te = hcd_v(c, HCD_X), *b = hcd_v(c, HCD_B);
  for (size_t q = 0; q < nc; ++q) {
    te[q] = gm * (pr[q] / ro[q]);
    b[q] = te[q];
  }
  hc_matrix(c, ro, te, bx, by, bz, dt, mat);
  const int ix = c->ix, jx = c->jx;
  const int is = p->margin[0], ie = ix - p->margin[0] - 1, js = p->margin[1], je = jx - p->margin[1] - 1;
  double *r = hcd_v(c, HCD_R), *r0 = hcd_v(c, HCD_R0), *pk = hcd_v(c, HCD_P);
  double a0 = 0.0, a1 = 0.0;
  for (int j = js; j <= je; ++j)
    for (int i = is; i <= ie; ++i) {
      const size_t q = (size_t)j * ix + i;
      double v = b[q];
      v = v - mat[q] * te[q];
      v = v - mat[q + nc] * te[q - 1];
      v = v - mat[q + 2 * nc] * te[q + 1];
      v = v - mat[q + 3 * nc] * te[q - ix];
      v = v - mat[q + 4 * nc] * te[q + ix];
      v = v - mat[q + 5 * nc] * te[q - 1 - ix];
      v = v - mat[q + 6 * nc] * te[q + 1 - ix];
      v = v - mat[q + 7 * nc] * te[q - 1 + ix];
      v = v - mat[q + 8 * nc] * te[q + 1 + ix];
      r[q] = v;
      r0[q] = v;
      pk[q] = v;
      a0 += v * v;
      a1 += b[q] * b[q];
    }
  sums[0] = a0;
  sums[1] = a1;
  return 0;
}

int orc_hcd_phase(orc_ctx *c, int phase, const double coef[2], double sums[2]) {
  const pip_params *p = &c->p;
  const size_t nc = c->nc;
  const int ix = c->ix, jx = c->jx;
  const int is = p->margin[0], ie = ix - p->margin[0] - 1, js = p->margin[1], je = jx - p->margin[1] - 1;
  const double *mat = hcd_v(c, HCD_NV);
  double *x = hcd_v(c, HCD_X), *b = hcd_v(c, HCD_B), *r = hcd_v(c, HCD_R), *r0 = hcd_v(c, HCD_R0);
  double *pk = hcd_v(c, HCD_P), *ap = hcd_v(c, HCD_AP), *t = hcd_v(c, HCD_T);
  double a0 = 0.0, a1 = 0.0;
  switch (phase) {
    case 0:
      for (size_t q = 0; q < nc; ++q) pk[q] = r[q];
      return 0;
    case 1:
      for (int j = js; j <= je; ++j)
        for (int i = is; i <= ie; ++i) {
          const size_t q = (size_t)j * ix + i;
          ap[q] = hc_apply(c, mat, pk, q);
          a0 = a0 + (r[q] * r0[q]);
          a1 = a1 + (r0[q] * ap[q]);
        }
      break;
    case 2:
      for (size_t q = 0; q < nc; ++q) t[q] = r[q] - coef[0] * ap[q];
      for (int j = js; j <= je; ++j)
        for (int i = is; i <= ie; ++i) {
          const size_t q = (size_t)j * ix + i;
          const double at = hc_apply(c, mat, t, q);
          a0 = a0 + t[q] * at;
          a1 = a1 + at * at;
        }
      break;
    case 3:
      for (size_t q = 0; q < nc; ++q) x[q] = x[q] + coef[0] * pk[q] + coef[1] * t[q];
      return 0;
    case 4:
      for (int j = js; j <= je; ++j)
        for (int i = is; i <= ie; ++i) {
          const size_t q = (size_t)j * ix + i;
          r[q] = b[q] - hc_apply(c, mat, x, q);
          a0 = a0 + r0[q] * r[q];
          a1 = a1 + r[q] * r[q];
        }
      break;
    case 5:
      for (size_t q = 0; q < nc; ++q) pk[q] = r[q] + coef[0] * (pk[q] - coef[1] * ap[q]);
      return 0;
    default:
      return PIP_ERR_PARAM;
  }
  sums[0] = a0;
  sums[1] = a1;
  return 0;
}

/* Row `row` of vector vec (0 x, 1 r, 2 Ap), ix values. */
void orc_hcd_get_row(const orc_ctx *c, int vec, int row, double *out) {
  const int k = vec == 0 ? HCD_X : vec == 1 ? HCD_R : HCD_AP;
  memcpy(out, hcd_v(c, k) + (size_t)row * c->ix, sizeof(double) * c->ix);
}
void orc_hcd_set_row(orc_ctx *c, int vec, int row, const double *in) {
  const int k = vec == 0 ? HCD_X : vec == 1 ? HCD_R : HCD_AP;
  memcpy(hcd_v(c, k) + (size_t)row * c->ix, in, sizeof(double) * c->ix);
}

int orc_hcd_end(orc_ctx *c) {
  const size_t nc = c->nc;
  const double gm = c->p.gm;
  const double *te = hcd_v(c, HCD_X), *w = hcd_v(c, HCD_NV) + 9 * nc;
  const double *ro = w, *vx = w + nc, *vy = w + 2 * nc, *vz = w + 3 * nc;
  const double *bx = w + 5 * nc, *by = w + 6 * nc, *bz = w + 7 * nc;
  double *U = c->U_m;
  for (size_t q = 0; q < nc; ++q) {
    const double pr = (te[q] * ro[q]) / gm;
    U[q] = ro[q];
    U[q + nc] = ro[q] * vx[q];
    U[q + 2 * nc] = ro[q] * vy[q];
    U[q + 3 * nc] = ro[q] * vz[q];
    U[q + 4 * nc] = pr / (gm - 1.0) + 0.5 * ro[q] * (vx[q] * vx[q] + vy[q] * vy[q] + vz[q] * vz[q]) +
                    0.5 * (bx[q] * bx[q] + by[q] * by[q] + bz[q] * bz[q]);
    U[q + 5 * nc] = bx[q];
    U[q + 6 * nc] = by[q];
    U[q + 7 * nc] = bz[q];
  }
  return 0;
}

/* One stage of run_solver, Solver_rot.f90:59-71 with set_flux :124, set_source :162,
 * time_integral :179-277 (flag_time=0), add_source :498-503, divb_cleaning_Dedner_source
 * (Scheme_rot.f90:546-554) and PIPbnd after the stage.  Stage 1 keeps U0 for stage 2. */
void orc_stage(orc_ctx *c, int istep, double dt) {
  const pip_params *p = &c->p;
  size_t nc = c->nc;
  int nh = c->nh, nm = c->nm, t_order = p->t_order;
  if (istep == 1) {
    ensure_coefficients(c);
    if (!c->U_h0) c->U_h0 = malloc(sizeof(double) * nc * nh);
    if (!c->U_m0) c->U_m0 = malloc(sizeof(double) * nc * nm);
    memcpy(c->U_h0, c->U_h, sizeof(double) * nc * nh);
    memcpy(c->U_m0, c->U_m, sizeof(double) * nc * nm);
    c->stage_dt = dt;
  }
  double *U_h0 = c->U_h0, *U_m0 = c->U_m0;
  double *F_h = calloc(nc * nh * 3, sizeof(double)), *F_m = calloc(nc * nm * 3, sizeof(double));
  double *S_h = malloc(sizeof(double) * nc * nh), *S_m = malloc(sizeof(double) * nc * nm);
  double dt_coll[2] = {dt * 0.5, dt * 0.5};
  double dt_coll_i = dt_coll[t_order - istep];
  /* set_coefficients(U_h,U_m,1) (Solver_rot.f90:62): flag_resi >= 2 recomputes eta
   * (:98-101), flag_col >= 2 alpha_c, flag_IR >= 2 the rates (after it, :108-112) */
  if (c->resi == 2) set_resistivity_anomalous(c);
  if (c->col_type >= 1) set_collisional(c);
  if (ir_per_stage(c)) set_ir_law(c);
  for (int dir = 1; dir <= p->ndim; ++dir)
    flux_dir(c, dir, F_h + (size_t)(dir - 1) * nc * nh, F_m + (size_t)(dir - 1) * nc * nm);
  memset(S_h, 0, sizeof(double) * nc * nh);
  memset(S_m, 0, sizeof(double) * nc * nm);
  source_pip(c, U_h0, U_m0, dt_coll_i, S_h, S_m);
  double dt_sub = dt / (double)(t_order - istep + 1);
  for (int dir = 1; dir <= p->ndim; ++dir)
    add_flux_rk(c, F_h + (size_t)(dir - 1) * nc * nh, U_h0, c->U_h, nh, dt_sub, dir);
  for (size_t q = 0; q < nc * nh; ++q) c->U_h[q] = c->U_h[q] + S_h[q] * dt_sub;
  for (int dir = 1; dir <= p->ndim; ++dir)
    add_flux_rk(c, F_m + (size_t)(dir - 1) * nc * nm, U_m0, c->U_m, nm, dt_sub, dir);
  for (size_t q = 0; q < nc * nm; ++q) c->U_m[q] = c->U_m[q] + S_m[q] * dt_sub;
  if (p->flag_divb == 1) {
    double fac = exp(-dt_sub / dt * p->safety * p->db_clean);
    double *ps = c->U_m + 8 * nc;
    for (size_t q = 0; q < nc; ++q) ps[q] = ps[q] * fac;
  }
  if (p->flag_ir == PIP_IR_NLEVEL) hydrogen_excitation_update(c, dt_sub);
  orc_bnd(c);
  free(F_h); free(F_m); free(S_h); free(S_m);
}

/* run_solver, Solver_rot.f90:42-81: t_order stages, then post_step's implicit conduction
 * of the ions (:296-303) and the closing PIPbnd. */
void orc_run_solver(orc_ctx *c, double dt) {
  for (int istep = 1; istep <= c->p.t_order; ++istep) orc_stage(c, istep, dt);
  if (c->p.flag_heat == 1) orc_conduction(c, dt, NULL, NULL);
  orc_bnd(c);
}

int orc_has_nan(const orc_ctx *c) {
  size_t nc = c->nc;
  int bad = 0;
  for (size_t q = 0; q < nc * c->nm; ++q) bad |= !isfinite(c->U_m[q]);
  for (size_t q = 0; q < nc * c->nh; ++q) bad |= !isfinite(c->U_h[q]);
  return bad;
}

/* Time loop, main.f90:31-68: set_IR and cfl, run_solver, cfl again, time += dt,
 * stop_sim (IO_rot.f90:625-674). */
int orc_run(orc_ctx *c, long nsteps, double t_end, double *time_out, long *steps_done,
            double *dt_hist, long max_hist) {
  long n = 0;
  int status = 0;
  while ((nsteps <= 0 || n < nsteps) && (t_end <= 0.0 || c->time < t_end)) {
    double dt, cmax, dtnew;
    orc_cfl(c, &dt, &cmax);
    c->cmax = cmax;
    orc_run_solver(c, dt);
    orc_cfl(c, &dtnew, NULL);
    /* the second cfl's cfl_resi lowers the global dt with the eta of the last stage (a
     * no-op for a fixed eta field, whose bound dt already holds) */
    if (c->resi) dt = cfl_resi(c, dt);
    c->time = c->time + dt;
    c->last_dt = dt;
    if (dt_hist && n < max_hist) dt_hist[n] = dt;
    ++n;
    if (orc_has_nan(c)) { status = PIP_ERR_NAN; break; }
    if (dt <= 1.0e-12) { status = PIP_ERR_DT; break; }
  }
  if (time_out) *time_out = c->time;
  if (steps_done) *steps_done = n;
  return status;
}

/* ---------------------------------------------------------------- lifecycle */

orc_ctx *orc_create(const pip_params *p, int *status) {
  *status = PIP_ERR_PARAM;
  if (!p || p->ndim < 1 || p->ndim > 2 || p->kx != 1 || p->nvar_h != 5) return NULL;
  if (p->nvar_m != (p->flag_divb == 1 ? 9 : 8)) return NULL;
  if (p->flag_heat == 1 && (p->ndim != 2 || p->hc_max < 0 || !(p->hc_error > 0.0))) return NULL;
  if (p->flag_col < 1 || p->flag_col > 7) return NULL;
  if (p->flag_resi < 0 || p->flag_resi > 2) return NULL;
  if (p->flag_resi == 2 && p->resi_type != 2 && p->resi_type != 3) return NULL;
  orc_ctx *c = calloc(1, sizeof(orc_ctx));
  c->p = *p;
  for (int f = 0; f < 6; ++f) c->neighbor[f] = -1;
  c->ix = p->ix; c->jx = p->jx; c->kx = p->kx;
  c->nh = p->nvar_h; c->nm = p->nvar_m;
  c->nc = (size_t)c->ix * c->jx * c->kx;
  c->dx = malloc(sizeof(double) * c->ix);
  c->dy = malloc(sizeof(double) * c->jx);
  c->dz = malloc(sizeof(double) * c->kx);
  memcpy(c->dx, p->dx, sizeof(double) * c->ix);
  memcpy(c->dy, p->dy, sizeof(double) * c->jx);
  memcpy(c->dz, p->dz, sizeof(double) * c->kx);
  c->U_h = calloc(c->nc * c->nh, sizeof(double));
  c->U_m = calloc(c->nc * c->nm, sizeof(double));
  c->gm_ion = calloc(c->nc, sizeof(double));
  c->gm_rec = calloc(c->nc, sizeof(double));
  c->col_type = p->flag_col >= 2 ? p->flag_col - 1 : 0;   /* PIP_rot.f90:21-26 */
  c->resi = p->flag_resi;
  if (c->resi) {
    c->eta = malloc(sizeof(double) * c->nc);
    for (size_t q = 0; q < c->nc; ++q) c->eta[q] = p->eta_0;   /* set_resistivity type 0 */
  }
  if (c->col_type >= 1) c->ac = calloc(c->nc, sizeof(double));
  set_sym_mhd(c);
  set_sym_hd(c);
  *status = PIP_OK;
  return c;
}

void orc_destroy(orc_ctx *c) {
  if (!c) return;
  free(c->dx); free(c->dy); free(c->dz);
  free(c->U_h); free(c->U_m); free(c->gm_ion); free(c->gm_rec);
  free(c->U_h0); free(c->U_m0);
  free(c->ac);
  free(c->eta);
  free(c->etab); free(c->nex); free(c->colrat); free(c->ion_pot);
  free(c->hcd);
  free(c);
}

void orc_set_state(orc_ctx *c, const double *U_h, const double *U_m) {
  memcpy(c->U_h, U_h, sizeof(double) * c->nc * c->nh);
  memcpy(c->U_m, U_m, sizeof(double) * c->nc * c->nm);
}

void orc_get_state(const orc_ctx *c, double *U_h, double *U_m) {
  memcpy(U_h, c->U_h, sizeof(double) * c->nc * c->nh);
  memcpy(U_m, c->U_m, sizeof(double) * c->nc * c->nm);
}

void orc_set_time(orc_ctx *c, double t) { c->time = t; }
double orc_get_time(const orc_ctx *c) { return c->time; }
double orc_get_cmax(const orc_ctx *c) { return c->cmax; }
void orc_set_cmax(orc_ctx *c, double cmax) { c->cmax = cmax; }
