/*
 * mg_oracle.c -- CPU FP64 restatement of the reference multigrid solver
 * (ANELASTIC_SL/mgMK).  TEST INFRASTRUCTURE ONLY: the parity tests, the
 * smoke check and the CPU-baseline leg of bench.py use it as the checker;
 * the product library never links or calls it.
 *
 * Serial semantics throughout: the reference's MPI halo exchange inside
 * mg_bdry becomes the full periodic wrap of the serial branch
 * (mg_bdry.F90:72-83), followed by the wall conditions.
 *
 * Arrays are stored as in the reference: one 1-D workspace per quantity,
 * levels packed finest first at kp3d(level) (mg_init.F90:194-220); inside a
 * level, (i,j,k) with 1-based ghosted indices s-1..e+1 maps to
 * (i-1) + X*((j-1) + Y*(k-1)), X = e_x+1, Y = e_y+1 (s = 2 on every level).
 *
 * Build: -O2 -ffp-contract=off (no FMA contraction, no reassociation).
 */
#include "oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ML (ANEL_MAX_LEVELS + 1)

struct orc_mg {
  int nx, ny, nz;
  double xL, yL, zL;
  int L[3], ngrid;
  int nk[ML][3];          /* nxk, nyk, nzk (= interior + 1) */
  int sk[ML][3], ek[ML][3];
  long kp3d[ML];          /* 1-based offsets into the 3-D workspaces */
  int kpx[ML][3];         /* 1-based offsets into the 1-D metric arrays */
  long nwork3d;
  int nworkx[3];
  double* workc[7];
  double* work1;
  double* work2;
  /* coarse metric hierarchy (mg_grids.F90), per direction */
  double* ek1[3];         /* xek */
  double* ck1[3];         /* xck */
  double* dck1[3];        /* dxck */
  double* dek1[3];        /* dxek */
  double* pcf[6];         /* pcf_1..pcf_6 (mg_coeff.F90) */
  /* METRIC mode hierarchy: per level and direction, local arrays
   * (index q-1 for the 1-based ghosted q) of E, C, DC, DE */
  double* ag[ML][3][4];
  int bd[27];
  double phibc[ML][6];
  int tbc[6];
  double vbc[6];
  int maxcy;
  double tolmax;
  int smoother, mode, stop;
  int pre[ML], post[ML];
  double* r;              /* Flow::r, fine ghosted */
  /* fine grid metrics, n+2 each, [0] = Fortran index 1 */
  double* fe[3];
  double* fc[3];
  double* fde[3];
  double* fdc[3];
  double* frde[3];
  double* frdc[3];
};

/* ---------------------------------------------------------------- helpers */

static inline long lvl_dim(const orc_mg* m, int l, int d) { return (long)m->ek[l][d] + 1; }
static inline long lvl_size(const orc_mg* m, int l) {
  return lvl_dim(m, l, 0) * lvl_dim(m, l, 1) * lvl_dim(m, l, 2);
}
/* 1-based ghosted (i,j,k) -> 0-based offset within a level block */
#define AT(a, i, j, k) (a)[((long)(i) - 1) + X * (((long)(j) - 1) + Y * ((long)(k) - 1))]
#define LVLDIMS(m, l)              \
  const long X = lvl_dim(m, l, 0); \
  const long Y = lvl_dim(m, l, 1); \
  (void)X;                         \
  (void)Y

static double* lvl_ptr(double* base, const orc_mg* m, int l) { return base + (m->kp3d[l] - 1); }

/* ------------------------------------------------------------ mg_check_size
 * mg_check_size.F90:77-151 (serial part: codes 4..6 and 10..12). */
static int check_size(const orc_mg* m, const int nC[3]) {
  const int nF[3] = {m->nx, m->ny, m->nz};
  for (int d = 0; d < 3; ++d) {
    if (nF[d] + 1 != nC[d] * (1 << (m->L[d] - 1)) + 1) return 4 + d;
  }
  if (m->ngrid > 1) {
    /* the ZLINE extension allows horizontal semi-coarsening (no z levels) */
    for (int d = 0; d < 3; ++d)
      if (m->L[d] == 1 && !(d == 2 && m->smoother == ANEL_SMOOTHER_ZLINE)) return 10 + d;
  }
  /* a single level would make mg_cycle restrict into level 0
   * (mg_cycle.F90:226); that is rejected here (code 13, not in the
   * reference). */
  if (m->ngrid < 2) return 13;
  return 0;
}

/* ---------------------------------------------------------------- mg_grids
 * mg_grids.F90:54-448 for one direction d (0=x,1=y,2=z).  tmin/tmax are
 * tbc of the min/max face of that direction. */
static void grids_dir(orc_mg* m, int d, int tmin, int tmax) {
  double* ek = m->ek1[d];
  double* ck = m->ck1[d];
  double* dck = m->dck1[d];
  double* dek = m->dek1[d];
  const int ng = m->ngrid;
  for (int q = 0; q < m->nworkx[d]; ++q) {
    dck[q] = 99999999999.0;
    dek[q] = 99999999999.0;
  }
  /* finest grid: copy of the fine metrics, Fortran 1..nxm+1 (:56-88) */
  const int nm = m->nk[ng][d];
  const int kx = m->kpx[ng][d];
  for (int i2 = 1; i2 <= nm + 1; ++i2) {
    const int i = i2 + kx - 1;
    ek[i - 1] = m->fe[d][i2 - 1];
    ck[i - 1] = m->fc[d][i2 - 1];
    dek[i - 1] = m->fde[d][i2 - 1];
    dck[i - 1] = m->fdc[d][i2 - 1];
  }
  const double LL = m->fe[d][nm] - m->fe[d][0]; /* xe(nxm+1)-xe(1) */
  const int Ld = m->L[d];
#define E(q) ek[(q) - 1]
#define C(q) ck[(q) - 1]
#define DC(q) dck[(q) - 1]
#define DE(q) dek[(q) - 1]
  for (int lvl = ng; lvl >= ng - Ld + 2; --lvl) {
    const int lF = lvl, lC = lvl - 1;
    const int nc = m->nk[lC][d];
    const int nf = m->nk[lF][d];
    const int kC = m->kpx[lC][d];
    const int kF = m->kpx[lF][d];
    if (tmin == 0) { /* periodic: uniform coarse spacing (:120-138) */
      const double dxx = LL / (double)nc;
      for (int i = 1; i <= nc + 1; ++i) E(i + kC - 1) = -dxx + dxx * (double)i;
      for (int i = 2; i <= nc + 1; ++i) {
        const int q = i + kC - 1;
        C(q) = (E(q) + E(q - 1)) / 2.0;
      }
      C(kC) = E(kC) - 0.5 * dxx;
      for (int i = 1; i <= nc + 1; ++i) {
        DC(i + kC - 1) = dxx;
        DE(i + kC - 1) = dxx;
      }
    } else { /* walls (:140-196) */
      int iif = kF, iic = kC;
      E(iic) = E(iif);
      for (int ic1 = 2; ic1 <= nc; ++ic1) {
        iif = (kF - 1) + 2 * ic1 - 2;
        iic = (kC - 1) + ic1;
        C(iic) = C(iif) + DC(iif) * 0.5;
        E(iic) = C(iic) + DC(iif);
      }
      iic = kC;
      iif = kF;
      if (tmin == 2) C(iic) = C(iif);
      else C(iic) = C(iif) - 0.5 * DE(iif + 1);
      iic = kC + nc;
      iif = kF + nf;
      if (tmax == 2) {
        C(iic) = C(iif);
        E(iic) = E(iif);
      } else {
        C(iic) = C(iif) + 0.5 * DE(iif - 1);
        E(iic) = E(iif) + 0.5 * DC(iif - 1);
      }
      for (int ic1 = 2; ic1 <= nc; ++ic1) {
        iic = (kC - 1) + ic1;
        DE(iic) = C(iic + 1) - C(iic);
        DC(iic) = E(iic) - E(iic - 1);
      }
      iic = kC;
      DC(iic) = 0.0;
      if (tmin == 2) DE(iic) = C(iic + 1) - C(iic);
      else DE(iic) = DE(iic + 1);
      iic = kC + nc;
      if (tmax == 2) {
        DE(iic) = C(iic) - C(iic - 1);
        DC(iic) = E(iic) - E(iic - 1);
      } else {
        DE(iic) = DE(iic - 1);
        DC(iic) = DC(iic - 1);
      }
    }
  }
  /* levels without coarsening in d copy the next finer level (:202-217) */
  for (int lvl = ng - Ld + 1; lvl >= 2; --lvl) {
    const int lF = lvl, lC = lvl - 1;
    const int nc = m->nk[lC][d];
    const int kC = m->kpx[lC][d], kF = m->kpx[lF][d];
    for (int i = 1; i <= nc + 1; ++i) {
      const int iif = (kF - 1) + i, iic = (kC - 1) + i;
      E(iic) = E(iif);
      C(iic) = C(iif);
      DE(iic) = DE(iif);
      DC(iic) = DC(iif);
    }
  }
#undef E
#undef C
#undef DC
#undef DE
}

/* mg_coeff.F90:77-145 for one level */
static void coeff_level(orc_mg* m, int lvl) {
  for (int d = 0; d < 3; ++d) {
    const int nm = m->nk[lvl][d];
    const int s = m->kpx[lvl][d]; /* 1-based start; local index q -> s+q-1 */
    double* pa = m->pcf[2 * d];
    double* pb = m->pcf[2 * d + 1];
    const double* de = m->dek1[d];
    const double* dc = m->dck1[d];
    for (int q = 2; q <= nm; ++q) {
      const long g = s + q - 1; /* 1-based global */
      const double west = de[g - 1 - 1];
      const double east = de[g - 1];
      pa[g - 1] = 1.0 / (dc[g - 1] * west);
      pb[g - 1] = 1.0 / (dc[g - 1] * east);
    }
  }
  if (lvl == m->ngrid) {
    const int* t = m->tbc;
    if (t[4] == 1) m->pcf[0][m->kpx[lvl][0] + 2 - 1 - 1] = 0.0;
    if (t[5] == 1) m->pcf[1][m->kpx[lvl][0] + m->nk[lvl][0] - 1 - 1] = 0.0;
    if (t[2] == 1) m->pcf[2][m->kpx[lvl][1] + 2 - 1 - 1] = 0.0;
    if (t[0] == 1) m->pcf[3][m->kpx[lvl][1] + m->nk[lvl][1] - 1 - 1] = 0.0;
    if (t[1] == 1) m->pcf[4][m->kpx[lvl][2] + 2 - 1 - 1] = 0.0;
    if (t[3] == 1) m->pcf[5][m->kpx[lvl][2] + m->nk[lvl][2] - 1 - 1] = 0.0;
  }
}
/* METRIC mode coarse metrics (a documented deviation): cell-centred
 * agglomeration.  Coarse edge q is fine edge 2q-1, coarse widths and
 * centres follow from the edges, ghost cells mirror their interior
 * neighbour.  Directions not coarsened copy the finer level. */
static void agglomerate(orc_mg* m) {
  const int ng = m->ngrid;
  for (int d = 0; d < 3; ++d) {
    const int nf = m->nk[ng][d] - 1;
    for (int a = 0; a < 4; ++a) m->ag[ng][d][a] = (double*)malloc(sizeof(double) * (nf + 2));
    memcpy(m->ag[ng][d][0], m->fe[d], sizeof(double) * (nf + 2));
    memcpy(m->ag[ng][d][1], m->fc[d], sizeof(double) * (nf + 2));
    memcpy(m->ag[ng][d][2], m->fdc[d], sizeof(double) * (nf + 2));
    memcpy(m->ag[ng][d][3], m->fde[d], sizeof(double) * (nf + 2));
    for (int l = ng - 1; l >= 1; --l) {
      const int n = m->nk[l][d] - 1;
      for (int a = 0; a < 4; ++a) m->ag[l][d][a] = (double*)malloc(sizeof(double) * (n + 2));
      double *E = m->ag[l][d][0], *C = m->ag[l][d][1], *DC = m->ag[l][d][2], *DE = m->ag[l][d][3];
      const double* Ef = m->ag[l + 1][d][0];
      if (m->nk[l][d] == m->nk[l + 1][d]) {
        for (int a = 0; a < 4; ++a) memcpy(m->ag[l][d][a], m->ag[l + 1][d][a], sizeof(double) * (n + 2));
        continue;
      }
      for (int q = 1; q <= n + 1; ++q) E[q - 1] = Ef[2 * q - 2];
      for (int q = 2; q <= n + 1; ++q) {
        DC[q - 1] = E[q - 1] - E[q - 2];
        C[q - 1] = 0.5 * (E[q - 1] + E[q - 2]);
      }
      DC[0] = DC[1];
      DC[n + 1] = DC[n];
      C[0] = E[0] - 0.5 * DC[0];
      E[n + 1] = E[n] + DC[n + 1];
      C[n + 1] = E[n] + 0.5 * DC[n + 1];
      for (int q = 1; q <= n + 1; ++q) DE[q - 1] = C[q] - C[q - 1];
      DE[n + 1] = DE[n];
      /* a direction whose finer spacings are one value is coarsened
       * exactly: every coarse spacing is twice it */
      const int nf2 = m->nk[l + 1][d] + 1;
      const double* DCf = m->ag[l + 1][d][2];
      const double* DEf = m->ag[l + 1][d][3];
      int uni = 1;
      for (int q = 1; q < nf2; ++q)
        if (!(DCf[q] == DCf[0] && DEf[q] == DCf[0])) uni = 0;
      if (uni && DEf[0] == DCf[0])
        for (int q = 0; q < n + 2; ++q) DC[q] = DE[q] = 2.0 * DCf[0];
    }
  }
}

/* pcf_d(i) for local (level) index i */
static inline double PCF(const orc_mg* m, int which, int lvl, int i) {
  const int d = which / 2;
  return m->pcf[which][m->kpx[lvl][d] - 1 + i - 1];
}

/* ------------------------------------------------------------------ create */
orc_mg* orc_mg_create(const anel_grid_desc* g, const anel_mg_params* p, int* stat) {
  orc_mg* m = (orc_mg*)calloc(1, sizeof(orc_mg));
  m->nx = g->nx;
  m->ny = g->ny;
  m->nz = g->nz;
  m->xL = g->xL;
  m->yL = g->yL;
  m->zL = g->zL;
  for (int d = 0; d < 3; ++d) m->L[d] = p->levels[d];
  m->maxcy = p->maxcy;
  m->tolmax = p->tolmax;
  m->smoother = p->smoother;
  m->mode = p->mode;
  m->stop = p->stop;
  for (int f = 0; f < 6; ++f) {
    m->tbc[f] = p->tbc[f];
    m->vbc[f] = p->vbc[f];
  }
  const int n[3] = {g->nx, g->ny, g->nz};
  const double* src[3][6] = {{g->xe, g->xc, g->dxe, g->dxc, g->rdxe, g->rdxc},
                             {g->ye, g->yc, g->dye, g->dyc, g->rdye, g->rdyc},
                             {g->ze, g->zc, g->dze, g->dzc, g->rdze, g->rdzc}};
  for (int d = 0; d < 3; ++d) {
    double** dst[6] = {m->fe, m->fc, m->fde, m->fdc, m->frde, m->frdc};
    for (int a = 0; a < 6; ++a) {
      dst[a][d] = (double*)malloc(sizeof(double) * (n[d] + 2));
      memcpy(dst[a][d], src[d][a], sizeof(double) * (n[d] + 2));
    }
  }
  /* mg_init.F90:86-89 */
  m->ngrid = m->L[0];
  if (m->L[1] > m->ngrid) m->ngrid = m->L[1];
  if (m->L[2] > m->ngrid) m->ngrid = m->L[2];
  const int ng = m->ngrid;
  for (int l = 1; l <= ng; ++l) {
    m->pre[l] = p->pre_relax[l - 1];
    m->post[l] = p->post_relax[l - 1];
  }
  int nC[3];
  for (int d = 0; d < 3; ++d) nC[d] = n[d] / (1 << (m->L[d] - 1));
  *stat = check_size(m, nC);
  if (*stat != 0) return m;
  /* level sizes (:125-129) */
  for (int l = 1; l <= ng; ++l)
    for (int d = 0; d < 3; ++d) {
      int e = l + m->L[d] - ng;
      if (e < 1) e = 1;
      m->nk[l][d] = nC[d] * (1 << (e - 1)) + 1;
    }
  /* start/end indices (:131-190) */
  for (int d = 0; d < 3; ++d) {
    m->sk[ng][d] = 2;
    m->ek[ng][d] = n[d] + 1;
  }
  for (int l = ng - 1; l >= 1; --l)
    for (int d = 0; d < 3; ++d) {
      if (m->nk[l][d] < m->nk[l + 1][d]) {
        m->sk[l][d] = m->sk[l + 1][d] / 2 + 1;
        m->ek[l][d] = (m->ek[l + 1][d] - 1) / 2 + 1;
      } else {
        m->sk[l][d] = m->sk[l + 1][d];
        m->ek[l][d] = m->ek[l + 1][d];
      }
    }
  /* workspace offsets, finest first (:194-220) */
  long kp3 = 1;
  int kx[3] = {1, 1, 1};
  for (int l = ng; l >= 1; --l) {
    m->kp3d[l] = kp3;
    for (int d = 0; d < 3; ++d) {
      m->kpx[l][d] = kx[d];
      kx[d] = m->kpx[l][d] + (m->nk[l][d] - 2 + 3);
    }
    kp3 = m->kp3d[l] + (long)(m->ek[l][0] - m->sk[l][0] + 3) * (m->ek[l][1] - m->sk[l][1] + 3) *
                           (m->ek[l][2] - m->sk[l][2] + 3);
  }
  m->nwork3d = kp3;
  for (int d = 0; d < 3; ++d) m->nworkx[d] = kx[d];
  for (int c = 0; c < 7; ++c) m->workc[c] = (double*)calloc(m->nwork3d, sizeof(double));
  m->work1 = (double*)calloc(m->nwork3d, sizeof(double));
  m->work2 = (double*)calloc(m->nwork3d, sizeof(double));
  for (int d = 0; d < 3; ++d) {
    m->ek1[d] = (double*)calloc(m->nworkx[d], sizeof(double));
    m->ck1[d] = (double*)calloc(m->nworkx[d], sizeof(double));
    m->dck1[d] = (double*)calloc(m->nworkx[d], sizeof(double));
    m->dek1[d] = (double*)calloc(m->nworkx[d], sizeof(double));
    m->pcf[2 * d] = (double*)calloc(m->nworkx[d], sizeof(double));
    m->pcf[2 * d + 1] = (double*)calloc(m->nworkx[d], sizeof(double));
  }
  /* mg_grids: x uses tbc(5)/tbc(6), y tbc(3)/tbc(1), z tbc(2)/tbc(4) */
  grids_dir(m, 0, m->tbc[4], m->tbc[5]);
  grids_dir(m, 1, m->tbc[2], m->tbc[0]);
  grids_dir(m, 2, m->tbc[1], m->tbc[3]);
  for (int l = 1; l <= ng; ++l) coeff_level(m, l);
  agglomerate(m);
  /* bdMG (:265-305): serial, the domain touches every face */
  memset(m->bd, 0, sizeof(m->bd));
  m->bd[9] = m->tbc[4];
  m->bd[18] = m->tbc[5];
  m->bd[5] = m->tbc[2];
  m->bd[1] = m->tbc[0];
  m->bd[3] = m->tbc[1];
  m->bd[7] = m->tbc[3];
  for (int f = 0; f < 6; ++f) {
    m->phibc[ng][f] = m->vbc[f];
    for (int l = ng - 1; l >= 1; --l) m->phibc[l][f] = 0.0;
  }
  for (int i = 1; i <= 26; ++i)
    if (m->bd[i] > 2 || m->bd[i] < 0) {
      *stat = -1;
      return m;
    }
  /* default density r == 1 */
  const long G = (long)(n[0] + 2) * (n[1] + 2) * (n[2] + 2);
  m->r = (double*)malloc(sizeof(double) * G);
  for (long q = 0; q < G; ++q) m->r[q] = 1.0;
  *stat = 0;
  return m;
}

void orc_mg_destroy(orc_mg* m) {
  if (!m) return;
  for (int c = 0; c < 7; ++c) free(m->workc[c]);
  free(m->work1);
  free(m->work2);
  for (int d = 0; d < 3; ++d) {
    free(m->ek1[d]);
    free(m->ck1[d]);
    free(m->dck1[d]);
    free(m->dek1[d]);
    free(m->pcf[2 * d]);
    free(m->pcf[2 * d + 1]);
    free(m->fe[d]);
    free(m->fc[d]);
    free(m->fde[d]);
    free(m->fdc[d]);
    free(m->frde[d]);
    free(m->frdc[d]);
  }
  for (int l = 1; l <= m->ngrid; ++l)
    for (int d = 0; d < 3; ++d)
      for (int a = 0; a < 4; ++a) free(m->ag[l][d][a]);
  free(m->r);
  free(m);
}

void orc_mg_set_density(orc_mg* m, const double* r) {
  const long G = (long)(m->nx + 2) * (m->ny + 2) * (m->nz + 2);
  memcpy(m->r, r, sizeof(double) * G);
}

int orc_mg_levels(const orc_mg* m, int* out, int cap) {
  for (int l = 1; l <= m->ngrid && l <= cap; ++l) {
    int* o = out + (l - 1) * 12;
    o[0] = m->nk[l][0];
    o[1] = m->nk[l][1];
    o[2] = m->nk[l][2];
    o[3] = m->sk[l][0];
    o[4] = m->ek[l][0];
    o[5] = m->sk[l][1];
    o[6] = m->ek[l][1];
    o[7] = m->sk[l][2];
    o[8] = m->ek[l][2];
    o[9] = (int)m->kp3d[l];
    o[10] = m->kpx[l][0];
    o[11] = m->kpx[l][1];
  }
  return m->ngrid;
}

/* -------------------------------------------------------- coefficients
 * Fine level: mgdpfpde (mg_pfpde.F90:35-60).  r is the fine ghosted
 * density; r(i,j,k) with fine 1-based indices. */
#define RF(i, j, k) m->r[((long)(i) - 1) + RX * (((long)(j) - 1) + RY * ((long)(k) - 1))]

static void pfpde(orc_mg* m) {
  const int l = m->ngrid;
  LVLDIMS(m, l);
  const long RX = m->nx + 2, RY = m->ny + 2;
  double* c[7];
  for (int q = 0; q < 7; ++q) c[q] = lvl_ptr(m->workc[q], m, l);
  const int nxf = m->nk[l][0], nyf = m->nk[l][1], nzf = m->nk[l][2];
  const double dlx = m->xL / (double)(float)(nxf - 1);
  const double todlxx = 1.0 / (dlx * dlx);
  const double dly = m->yL / (double)(float)(nyf - 1);
  const double todlyy = 1.0 / (dly * dly);
  const double dlz = m->zL / (double)(float)(nzf - 1);
  const double todlzz = 1.0 / (dlz * dlz);
  for (int k = m->sk[l][2]; k <= m->ek[l][2]; ++k)
    for (int j = m->sk[l][1]; j <= m->ek[l][1]; ++j)
      for (int i = m->sk[l][0]; i <= m->ek[l][0]; ++i) {
        const double c1 = todlxx, c2 = todlxx, c3 = todlyy, c4 = todlyy;
        const double c5 = todlzz * 0.5 * (RF(i, j, k) + RF(i, j, k - 1)) / RF(i, j, k - 1);
        const double c6 = todlzz * 0.5 * (RF(i, j, k) + RF(i, j, k + 1)) / RF(i, j, k + 1);
        AT(c[0], i, j, k) = c1;
        AT(c[1], i, j, k) = c2;
        AT(c[2], i, j, k) = c3;
        AT(c[3], i, j, k) = c4;
        AT(c[4], i, j, k) = c5;
        AT(c[5], i, j, k) = c6;
        AT(c[6], i, j, k) =
            -(c1 + c2 + c3 + c4 + (todlzz * 0.5 * (RF(i, j, k) + RF(i, j, k - 1)) / RF(i, j, k)) +
              (todlzz * 0.5 * (RF(i, j, k) + RF(i, j, k + 1)) / RF(i, j, k)));
      }
}

/* The reference reads r one plane below its allocation at k = szm
 * (ks-1 = 0 at mg_phpde.F90:139); that read is undefined behaviour in the
 * reference.  Here the index is clamped to the ghost plane; the result is
 * overwritten by the wall zeroing whenever the z-min face is Neumann. */
static inline double r_clamped(const orc_mg* m, int i, int j, int k) {
  const long RX = m->nx + 2, RY = m->ny + 2;
  if (k < 1) k = 1;
  return RF(i, j, k);
}

/* Coarse levels: mgdphpde (mg_phpde.F90:111-199), including the stale
 * is/js/ks of the diagonal loop (:193-199). */
static void phpde(orc_mg* m, int l) {
  LVLDIMS(m, l);
  const int ng = m->ngrid;
  double* c[7];
  for (int q = 0; q < 7; ++q) c[q] = lvl_ptr(m->workc[q], m, l);
  const int nxm = m->nk[l][0], nym = m->nk[l][1], nzm = m->nk[l][2];
  const int nxf = m->nk[ng][0], nyf = m->nk[ng][1], nzf = m->nk[ng][2];
  const double dlx = m->xL / (double)(float)(nxm - 1);
  const double eidlxx = 1.0 / (dlx * dlx);
  const double dly = m->yL / (double)(float)(nym - 1);
  const double eidlyy = 1.0 / (dly * dly);
  const double dlz = m->zL / (double)(float)(nzm - 1);
  const double eidlzz = 1.0 / (dlz * dlz);
  const int istep = (nxf - 1) / (nxm - 1);
  const int jstep = (nyf - 1) / (nym - 1);
  const int kstep = (nzf - 1) / (nzm - 1);
  int is = 0, js = 0, ks = 0;
  const int sxm = m->sk[l][0], exm = m->ek[l][0];
  const int sym = m->sk[l][1], eym = m->ek[l][1];
  const int szm = m->sk[l][2], ezm = m->ek[l][2];
  for (int k = szm; k <= ezm; ++k) {
    const int km = 2 * kstep * k - 3 * (kstep - 1);
    for (int j = sym; j <= eym; ++j) {
      const int jm = 2 * jstep * j - 3 * (jstep - 1);
      for (int i = sxm; i <= exm; ++i) {
        const int im = 2 * istep * i - 3 * (istep - 1);
        is = (im - istep) / 2;
        js = jm / 2;
        ks = km / 2;
        AT(c[0], i, j, k) = eidlxx;
        is = (im + istep) / 2;
        AT(c[1], i, j, k) = eidlxx;
        is = im / 2;
        js = (jm - jstep) / 2;
        AT(c[2], i, j, k) = eidlyy;
        js = (jm - jstep) / 2;
        AT(c[3], i, j, k) = eidlyy;
        js = jm / 2;
        ks = (km - kstep) / 2;
        AT(c[4], i, j, k) = eidlzz * 0.5 * (r_clamped(m, is, js, ks) + r_clamped(m, is, js, ks - 1)) /
                            r_clamped(m, is, js, ks - 1);
        ks = (km + kstep) / 2;
        AT(c[5], i, j, k) = eidlzz * 0.5 * (r_clamped(m, is, js, ks) + r_clamped(m, is, js, ks + 1)) /
                            r_clamped(m, is, js, ks + 1);
      }
    }
  }
  const int* bd = m->bd;
  if (bd[1] == 1)
    for (int k = szm; k <= ezm; ++k)
      for (int i = sxm; i <= exm; ++i) AT(c[3], i, eym, k) = 0.0;
  if (bd[3] == 1)
    for (int j = sym; j <= eym; ++j)
      for (int i = sxm; i <= exm; ++i) AT(c[4], i, j, szm) = 0.0;
  if (bd[5] == 1)
    for (int k = szm; k <= ezm; ++k)
      for (int i = sxm; i <= exm; ++i) AT(c[2], i, sym, k) = 0.0;
  if (bd[7] == 1)
    for (int j = sym; j <= eym; ++j)
      for (int i = sxm; i <= exm; ++i) AT(c[5], i, j, ezm) = 0.0;
  if (bd[9] == 1)
    for (int k = szm; k <= ezm; ++k)
      for (int j = sym; j <= eym; ++j) AT(c[0], sxm, j, k) = 0.0;
  if (bd[18] == 1)
    for (int k = szm; k <= ezm; ++k)
      for (int j = sym; j <= eym; ++j) AT(c[1], exm, j, k) = 0.0;
  const double d5 = (eidlzz * 0.5 * (r_clamped(m, is, js, ks) + r_clamped(m, is, js, ks - 1)) /
                     r_clamped(m, is, js, ks));
  const double d6 = (eidlzz * 0.5 * (r_clamped(m, is, js, ks) + r_clamped(m, is, js, ks + 1)) /
                     r_clamped(m, is, js, ks));
  for (int k = szm; k <= ezm; ++k)
    for (int j = sym; j <= eym; ++j)
      for (int i = sxm; i <= exm; ++i)
        AT(c[6], i, j, k) = -(AT(c[0], i, j, k) + AT(c[1], i, j, k) + AT(c[2], i, j, k) +
                              AT(c[3], i, j, k) + d5 + d6);
}

/* METRIC mode (a documented deviation from the reference): every level's
 * operator is the 7-point stencil of the stretched metric.  Fine level:
 * rdxc(i)*rdxe(i-1) etc., i.e. exactly Psource(Pgrad(.)) of
 * NSsolver.F90:2060-2078,2212-2214 with r == 1; coarse levels:
 * 1/(dxc*dxe) products (the form of mg_coeff.F90:77-99) on the
 * agglomerated hierarchy of agglomerate() -- the reference's mg_grids
 * recursion drifts on strongly stretched grids and makes the V-cycle
 * diverge there.  Neumann faces zero the wall
 * coefficient on every level and the diagonal is minus the sum of the six
 * off-diagonals, so the operator is the consistent Neumann operator.
 * The density factors are those of the literal fine formula, evaluated
 * per cell (no stale index). */
static void metric_level(orc_mg* m, int l) {
  LVLDIMS(m, l);
  const int ng = m->ngrid;
  double* c[7];
  for (int q = 0; q < 7; ++q) c[q] = lvl_ptr(m->workc[q], m, l);
  const int sxm = m->sk[l][0], exm = m->ek[l][0];
  const int sym = m->sk[l][1], eym = m->ek[l][1];
  const int szm = m->sk[l][2], ezm = m->ek[l][2];
  const int nxf = m->nk[ng][0], nyf = m->nk[ng][1], nzf = m->nk[ng][2];
  const int istep = (nxf - 1) / (m->nk[l][0] - 1);
  const int jstep = (nyf - 1) / (m->nk[l][1] - 1);
  const int kstep = (nzf - 1) / (m->nk[l][2] - 1);
  for (int k = szm; k <= ezm; ++k)
    for (int j = sym; j <= eym; ++j)
      for (int i = sxm; i <= exm; ++i) {
        double a1, a2, a3, a4, a5, a6;
        if (l == ng) {
          a1 = m->frdc[0][i - 1] * m->frde[0][i - 2];
          a2 = m->frdc[0][i - 1] * m->frde[0][i - 1];
          a3 = m->frdc[1][j - 1] * m->frde[1][j - 2];
          a4 = m->frdc[1][j - 1] * m->frde[1][j - 1];
          a5 = m->frdc[2][k - 1] * m->frde[2][k - 2];
          a6 = m->frdc[2][k - 1] * m->frde[2][k - 1];
        } else {
          double* const* X_ = m->ag[l][0];
          double* const* Y_ = m->ag[l][1];
          double* const* Z_ = m->ag[l][2];
          a1 = 1.0 / (X_[2][i - 1] * X_[3][i - 2]);
          a2 = 1.0 / (X_[2][i - 1] * X_[3][i - 1]);
          a3 = 1.0 / (Y_[2][j - 1] * Y_[3][j - 2]);
          a4 = 1.0 / (Y_[2][j - 1] * Y_[3][j - 1]);
          a5 = 1.0 / (Z_[2][k - 1] * Z_[3][k - 2]);
          a6 = 1.0 / (Z_[2][k - 1] * Z_[3][k - 1]);
        }
        if (m->bd[9] == 1 && i == sxm) a1 = 0.0;
        if (m->bd[18] == 1 && i == exm) a2 = 0.0;
        if (m->bd[5] == 1 && j == sym) a3 = 0.0;
        if (m->bd[1] == 1 && j == eym) a4 = 0.0;
        if (m->bd[3] == 1 && k == szm) a5 = 0.0;
        if (m->bd[7] == 1 && k == ezm) a6 = 0.0;
        /* density: fine-level indices of this coarse cell's centre column */
        const int im = 2 * istep * i - 3 * (istep - 1);
        const int jm = 2 * jstep * j - 3 * (jstep - 1);
        const int km = 2 * kstep * k - 3 * (kstep - 1);
        const int fi = (l == ng) ? i : im / 2;
        const int fj = (l == ng) ? j : jm / 2;
        const int fk = (l == ng) ? k : km / 2;
        const double rp = r_clamped(m, fi, fj, fk);
        const double rb = r_clamped(m, fi, fj, fk - 1);
        const double rt = r_clamped(m, fi, fj, fk + 1);
        const double w5 = 0.5 * (rp + rb);
        const double w6 = 0.5 * (rp + rt);
        const double c5 = a5 * w5 / rb;
        const double c6 = a6 * w6 / rt;
        AT(c[0], i, j, k) = a1;
        AT(c[1], i, j, k) = a2;
        AT(c[2], i, j, k) = a3;
        AT(c[3], i, j, k) = a4;
        AT(c[4], i, j, k) = c5;
        AT(c[5], i, j, k) = c6;
        AT(c[6], i, j, k) = -(a1 + a2 + a3 + a4 + a5 * w5 / rp + a6 * w6 / rp);
      }
}

static void build_coeffs(orc_mg* m) {
  if (m->mode == ANEL_MODE_METRIC) {
    for (int l = m->ngrid; l >= 1; --l) metric_level(m, l);
    return;
  }
  pfpde(m);
  for (int l = m->ngrid - 1; l >= 1; --l) phpde(m, l);
}

/* ----------------------------------------------------------------- mg_bdry
 * mg_bdry.F90:1-192, serial branch: periodic wrap of all six faces, then
 * the wall conditions in the order X2max, X3min, X2min, X3max, X1min,
 * X1max.  The spacing arrays are indexed without the level offset, as in
 * the reference (dyck(eym) etc.); only the finest level has phibc != 0. */
static void bdry(orc_mg* m, int l, double* phi) {
  LVLDIMS(m, l);
  const long Z = lvl_dim(m, l, 2);
  const int sxm = m->sk[l][0], exm = m->ek[l][0];
  const int sym = m->sk[l][1], eym = m->ek[l][1];
  const int szm = m->sk[l][2], ezm = m->ek[l][2];
  const double* v = m->phibc[l];
  for (long k = 1; k <= Z; ++k)
    for (long j = 1; j <= Y; ++j) {
      AT(phi, sxm - 1, j, k) = AT(phi, exm, j, k);
      AT(phi, exm + 1, j, k) = AT(phi, sxm, j, k);
    }
  for (long k = 1; k <= Z; ++k)
    for (long i = 1; i <= X; ++i) {
      AT(phi, i, sym - 1, k) = AT(phi, i, eym, k);
      AT(phi, i, eym + 1, k) = AT(phi, i, sym, k);
    }
  for (long j = 1; j <= Y; ++j)
    for (long i = 1; i <= X; ++i) {
      AT(phi, i, j, szm - 1) = AT(phi, i, j, ezm);
      AT(phi, i, j, ezm + 1) = AT(phi, i, j, szm);
    }
  const double* dyck = m->dck1[1];
  const double* dzck = m->dck1[2];
  const double* dxck = m->dck1[0];
  const int* bd = m->bd;
  if (bd[1] == 1) {
    for (int k = szm - 1; k <= ezm + 1; ++k)
      for (int i = sxm - 1; i <= exm + 1; ++i)
        AT(phi, i, eym + 1, k) = AT(phi, i, eym, k) + v[0] * dyck[eym - 1];
  } else if (bd[1] == 2) {
    for (int k = szm - 1; k <= ezm + 1; ++k)
      for (int i = sxm - 1; i <= exm + 1; ++i) AT(phi, i, eym + 1, k) = v[0];
  }
  if (bd[3] == 1) {
    for (int j = sym - 1; j <= eym + 1; ++j)
      for (int i = sxm - 1; i <= exm + 1; ++i)
        AT(phi, i, j, szm - 1) = AT(phi, i, j, szm) - v[1] * dzck[szm - 1];
  } else if (bd[3] == 2) {
    for (int j = sym - 1; j <= eym + 1; ++j)
      for (int i = sxm - 1; i <= exm + 1; ++i) AT(phi, i, j, szm - 1) = v[1];
  }
  if (bd[5] == 1) {
    for (int k = szm - 1; k <= ezm + 1; ++k)
      for (int i = sxm - 1; i <= exm + 1; ++i)
        AT(phi, i, sym - 1, k) = AT(phi, i, sym, k) - v[2] * dyck[sym - 1];
  } else if (bd[5] == 2) {
    for (int k = szm - 1; k <= ezm + 1; ++k)
      for (int i = sxm - 1; i <= exm + 1; ++i) AT(phi, i, sym - 1, k) = v[2];
  }
  if (bd[7] == 1) {
    for (int j = sym - 1; j <= eym + 1; ++j)
      for (int i = sxm - 1; i <= exm + 1; ++i)
        AT(phi, i, j, ezm + 1) = AT(phi, i, j, ezm) + v[3] * dzck[ezm - 1];
  } else if (bd[7] == 2) {
    for (int j = sym - 1; j <= eym + 1; ++j)
      for (int i = sxm - 1; i <= exm + 1; ++i) AT(phi, i, j, ezm + 1) = v[3];
  }
  if (bd[9] == 1) {
    for (int k = szm - 1; k <= ezm + 1; ++k)
      for (int j = sym - 1; j <= eym + 1; ++j)
        AT(phi, sxm - 1, j, k) = AT(phi, sxm, j, k) - v[4] * dxck[sxm - 1];
  } else if (bd[9] == 2) {
    for (int k = szm - 1; k <= ezm + 1; ++k)
      for (int j = sym - 1; j <= eym + 1; ++j) AT(phi, sxm - 1, j, k) = v[4];
  }
  if (bd[18] == 1) {
    for (int k = szm - 1; k <= ezm + 1; ++k)
      for (int j = sym - 1; j <= eym + 1; ++j)
        AT(phi, exm + 1, j, k) = AT(phi, exm, j, k) + v[5] * dxck[exm - 1];
  } else if (bd[18] == 2) {
    for (int k = szm - 1; k <= ezm + 1; ++k)
      for (int j = sym - 1; j <= eym + 1; ++j) AT(phi, exm + 1, j, k) = v[5];
  }
}

/* ---------------------------------------------------------- mg_relaxRB
 * mg_relax.F90:133-178.  Pass 1 updates (i+j+k) even, pass 2 odd (s=2). */
static void relax_rb(orc_mg* m, int l, double* phi, const double* src, int iters) {
  LVLDIMS(m, l);
  double* c[7];
  for (int q = 0; q < 7; ++q) c[q] = lvl_ptr(m->workc[q], m, l);
  const int sxm = m->sk[l][0], exm = m->ek[l][0];
  const int sym = m->sk[l][1], eym = m->ek[l][1];
  const int szm = m->sk[l][2], ezm = m->ek[l][2];
  for (int it = 1; it <= iters; ++it) {
    for (int ipass = 1; ipass <= 2; ++ipass) {
      /* The reference toggles rb per j and per k starting from mod(sxm,2)
       * (pass 1) or 1-mod(sxm,2) (pass 2); the start of row (j,k) is
       * therefore sxm + (rb0 + (j-sym) + (k-szm)) mod 2.  Within a pass
       * every update reads only the other colour and ghosts, so the rows
       * are independent and may run in parallel. */
      const int rb0 = (ipass == 1) ? sxm % 2 : 1 - sxm % 2;
#pragma omp parallel for schedule(static)
      for (int k = szm; k <= ezm; ++k) {
        for (int j = sym; j <= eym; ++j) {
          const int rb = (rb0 + (j - sym) + (k - szm)) & 1;
          for (int i = sxm + rb; i <= exm; i += 2) {
            const double pcfsum = AT(c[6], i, j, k);
            AT(phi, i, j, k) =
                (AT(src, i, j, k) -
                 (AT(c[0], i, j, k) * AT(phi, i - 1, j, k) + AT(c[1], i, j, k) * AT(phi, i + 1, j, k) +
                  AT(c[2], i, j, k) * AT(phi, i, j - 1, k) + AT(c[3], i, j, k) * AT(phi, i, j + 1, k) +
                  AT(c[4], i, j, k) * AT(phi, i, j, k - 1) + AT(c[5], i, j, k) * AT(phi, i, j, k + 1))) /
                pcfsum;
          }
        }
      }
      bdry(m, l, phi);
    }
  }
  bdry(m, l, phi);
}

/* --------------------------------------------------- Thomas / relaxLz
 * mg_relax.F90:541-595 (a, b overwritten, c untouched) */
static void thomas(double* a, double* b, const double* c, double* G, int n) {
  for (int j = 1; j <= n - 1; ++j) {
    a[j] = -a[j] / b[j - 1];
    b[j] = b[j] + a[j] * c[j - 1];
    G[j] = G[j] + a[j] * G[j - 1];
  }
  G[n - 1] = G[n - 1] / b[n - 1];
  for (int j = n - 1; j >= 1; --j) G[j - 1] = (G[j - 1] - c[j - 1] * G[j]) / b[j - 1];
}

/* mg_relaxLz (mg_relax.F90:423-538): (i+j) red-black z-line Gauss-Seidel
 * with the pcf_* metric coefficients. */
static void relax_lz(orc_mg* m, int l, double* phi, const double* src, int iters) {
  LVLDIMS(m, l);
  const int sxm = m->sk[l][0], exm = m->ek[l][0];
  const int sym = m->sk[l][1], eym = m->ek[l][1];
  const int szm = m->sk[l][2], ezm = m->ek[l][2];
  const int n = ezm - szm + 1;
  double* a = (double*)malloc(sizeof(double) * n);
  double* b = (double*)malloc(sizeof(double) * n);
  double* c = (double*)malloc(sizeof(double) * n);
  double* rhs = (double*)malloc(sizeof(double) * n);
  for (int k = szm; k <= ezm; ++k) c[k - szm] = PCF(m, 5, l, k);
  for (int it = 1; it <= iters; ++it) {
    int rb = sxm % 2;
    for (int ipass = 1; ipass <= 2; ++ipass) {
      for (int j = sym; j <= eym; ++j) {
        for (int i = sxm + rb; i <= exm; i += 2) {
          const double p1 = PCF(m, 0, l, i), p2 = PCF(m, 1, l, i);
          const double p3 = PCF(m, 2, l, j), p4 = PCF(m, 3, l, j);
          for (int k = szm; k <= ezm; ++k) {
            a[k - szm] = PCF(m, 4, l, k);
            b[k - szm] = -(p1 + p2 + p3 + p4 + PCF(m, 4, l, k) + PCF(m, 5, l, k));
          }
          for (int k = szm + 1; k <= ezm - 1; ++k)
            rhs[k - szm] = AT(src, i, j, k) - (p1 * AT(phi, i - 1, j, k) + p2 * AT(phi, i + 1, j, k) +
                                               p3 * AT(phi, i, j - 1, k) + p4 * AT(phi, i, j + 1, k));
          rhs[0] = AT(src, i, j, szm) -
                   (p1 * AT(phi, i - 1, j, szm) + p2 * AT(phi, i + 1, j, szm) + p3 * AT(phi, i, j - 1, szm) +
                    p4 * AT(phi, i, j + 1, szm) + PCF(m, 4, l, szm) * AT(phi, i, j, szm - 1));
          rhs[n - 1] = AT(src, i, j, ezm) -
                       (p1 * AT(phi, i - 1, j, ezm) + p2 * AT(phi, i + 1, j, ezm) +
                        p3 * AT(phi, i, j - 1, ezm) + p4 * AT(phi, i, j + 1, ezm) +
                        PCF(m, 5, l, ezm) * AT(phi, i, j, ezm + 1));
          thomas(a, b, c, rhs, n);
          for (int k = szm; k <= ezm; ++k) AT(phi, i, j, k) = rhs[k - szm];
        }
        rb = 1 - rb;
      }
      rb = 1 - sxm % 2;
      bdry(m, l, phi);
    }
  }
  bdry(m, l, phi);
  free(a);
  free(b);
  free(c);
  free(rhs);
}

/* ZLINE smoother (an extension, not in the reference): (i+j) red-black
 * z-line Gauss-Seidel with the level's own 7-point coefficients (the
 * operator the residual uses), each line solved by the Thomas algorithm of
 * mg_relax.F90:541-595; boundary pass after each colour. */
static void relax_zl(orc_mg* m, int l, double* phi, const double* src, int iters) {
  LVLDIMS(m, l);
  double* c[7];
  for (int q = 0; q < 7; ++q) c[q] = lvl_ptr(m->workc[q], m, l);
  const int sxm = m->sk[l][0], exm = m->ek[l][0];
  const int sym = m->sk[l][1], eym = m->ek[l][1];
  const int szm = m->sk[l][2], ezm = m->ek[l][2];
  const int n = ezm - szm + 1;
  for (int it = 1; it <= iters; ++it) {
    for (int ipass = 1; ipass <= 2; ++ipass) {
      const int rb0 = (ipass == 1) ? 0 : 1;
#pragma omp parallel for schedule(static)
      for (int j = sym; j <= eym; ++j) {
        double* a = (double*)malloc(sizeof(double) * 4 * n);
        double* b = a + n;
        double* cc = b + n;
        double* rhs = cc + n;
        const int rb = (rb0 + (j - sym)) & 1;
        for (int i = sxm + rb; i <= exm; i += 2) {
          for (int k = szm; k <= ezm; ++k) {
            const int q = k - szm;
            a[q] = AT(c[4], i, j, k);
            b[q] = AT(c[6], i, j, k);
            cc[q] = AT(c[5], i, j, k);
            rhs[q] = AT(src, i, j, k) -
                     (AT(c[0], i, j, k) * AT(phi, i - 1, j, k) + AT(c[1], i, j, k) * AT(phi, i + 1, j, k) +
                      AT(c[2], i, j, k) * AT(phi, i, j - 1, k) + AT(c[3], i, j, k) * AT(phi, i, j + 1, k));
          }
          rhs[0] = rhs[0] - a[0] * AT(phi, i, j, szm - 1);
          rhs[n - 1] = rhs[n - 1] - cc[n - 1] * AT(phi, i, j, ezm + 1);
          thomas(a, b, cc, rhs, n);
          for (int k = szm; k <= ezm; ++k) AT(phi, i, j, k) = rhs[k - szm];
        }
        free(a);
      }
      bdry(m, l, phi);
    }
  }
  bdry(m, l, phi);
}

static void relax(orc_mg* m, int l, double* phi, const double* src, int iters) {
  if (m->smoother == ANEL_SMOOTHER_LJ) relax_lz(m, l, phi, src, iters);
  else if (m->smoother == ANEL_SMOOTHER_ZLINE) relax_zl(m, l, phi, src, iters);
  else relax_rb(m, l, phi, src, iters);
}

/* --------------------------------------------------------------- mg_restr
 * mg_restr.F90:114-241.  res is the caller's rhsf buffer reinterpreted
 * with level lF's shape (mg_cycle.F90:226-227). */
static void restr(orc_mg* m, int lC, int lF, double* res) {
  double* phic = lvl_ptr(m->work1, m, lC);
  double* rhsc = lvl_ptr(m->work2, m, lC);
  const double* phif = lvl_ptr(m->work1, m, lF);
  const double* srcf = lvl_ptr(m->work2, m, lF);
  double* c[7];
  for (int q = 0; q < 7; ++q) c[q] = lvl_ptr(m->workc[q], m, lF);
  const long Gc = lvl_size(m, lC);
  for (long q = 0; q < Gc; ++q) {
    phic[q] = 0.0;
    rhsc[q] = 0.0;
  }
  {
    LVLDIMS(m, lF);
    const long Gf = lvl_size(m, lF);
    for (long q = 0; q < Gf; ++q) res[q] = 0.0;
#pragma omp parallel for schedule(static)
    for (int k = m->sk[lF][2]; k <= m->ek[lF][2]; ++k)
      for (int j = m->sk[lF][1]; j <= m->ek[lF][1]; ++j)
        for (int i = m->sk[lF][0]; i <= m->ek[lF][0]; ++i)
          AT(res, i, j, k) =
              AT(srcf, i, j, k) -
              (AT(c[0], i, j, k) * AT(phif, i - 1, j, k) + AT(c[1], i, j, k) * AT(phif, i + 1, j, k) +
               AT(c[2], i, j, k) * AT(phif, i, j - 1, k) + AT(c[3], i, j, k) * AT(phif, i, j + 1, k) +
               AT(c[4], i, j, k) * AT(phif, i, j, k - 1) + AT(c[5], i, j, k) * AT(phif, i, j, k + 1) +
               AT(c[6], i, j, k) * AT(phif, i, j, k));
  }
  const long XF = lvl_dim(m, lF, 0), YF = lvl_dim(m, lF, 1);
  const long XC = lvl_dim(m, lC, 0), YC = lvl_dim(m, lC, 1);
#define RS(i, j, k) res[((long)(i) - 1) + XF * (((long)(j) - 1) + YF * ((long)(k) - 1))]
#define RC(i, j, k) rhsc[((long)(i) - 1) + XC * (((long)(j) - 1) + YC * ((long)(k) - 1))]
  const int nxc = m->nk[lC][0], nyc = m->nk[lC][1], nzc = m->nk[lC][2];
  const int nxf = m->nk[lF][0], nyf = m->nk[lF][1], nzf = m->nk[lF][2];
  const int sxc = m->sk[lC][0], exc = m->ek[lC][0];
  const int syc = m->sk[lC][1], eyc = m->ek[lC][1];
  const int szc = m->sk[lC][2], ezc = m->ek[lC][2];
  if (nxc < nxf && nyc < nyf && nzc < nzf) {
#pragma omp parallel for schedule(static)
    for (int kc = szc; kc <= ezc; ++kc) {
      const int k = 2 * kc - 2;
      for (int jc = syc; jc <= eyc; ++jc) {
        const int j = 2 * jc - 2;
        for (int ic = sxc; ic <= exc; ++ic) {
          const int i = 2 * ic - 2;
          RC(ic, jc, kc) = 0.125 * (RS(i, j, k) + RS(i, j + 1, k) + RS(i, j, k + 1) + RS(i, j + 1, k + 1) +
                                    RS(i + 1, j, k) + RS(i + 1, j + 1, k + 1) + RS(i + 1, j + 1, k) +
                                    RS(i + 1, j, k + 1));
        }
      }
    }
  } else if (nxf == nxc && nyf == nyc) {
    for (int kc = szc; kc <= ezc; ++kc)
      for (int jc = syc; jc <= eyc; ++jc)
        for (int ic = sxc; ic <= exc; ++ic) {
          const int k = 2 * kc - 2;
          RC(ic, jc, kc) = 0.5 * (RS(ic, jc, k) + RS(ic, jc, k + 1));
        }
  } else if (nxf == nxc && nzf == nzc) {
    for (int kc = szc; kc <= ezc; ++kc)
      for (int jc = syc; jc <= eyc; ++jc)
        for (int ic = sxc; ic <= exc; ++ic) {
          const int j = 2 * jc - 2;
          RC(ic, jc, kc) = 0.5 * (RS(ic, j, kc) + RS(ic, j + 1, kc));
        }
  } else if (nyf == nyc && nzf == nzc) {
    for (int kc = szc; kc <= ezc; ++kc)
      for (int jc = syc; jc <= eyc; ++jc)
        for (int ic = sxc; ic <= exc; ++ic) {
          const int i = 2 * ic - 2;
          RC(ic, jc, kc) = 0.5 * (RS(i, jc, kc) + RS(i + 1, jc, kc));
        }
  } else if (nxf == nxc) {
    for (int kc = szc; kc <= ezc; ++kc)
      for (int jc = syc; jc <= eyc; ++jc)
        for (int ic = sxc; ic <= exc; ++ic) {
          const int k = 2 * kc - 2, j = 2 * jc - 2, i = ic;
          RC(ic, jc, kc) = 0.25 * (RS(i, j, k) + RS(i, j + 1, k) + RS(i, j, k + 1) + RS(i, j + 1, k + 1));
        }
  } else if (nyf == nyc) {
    for (int kc = szc; kc <= ezc; ++kc)
      for (int jc = syc; jc <= eyc; ++jc)
        for (int ic = sxc; ic <= exc; ++ic) {
          const int k = 2 * kc - 2, j = jc, i = 2 * ic - 2;
          RC(ic, jc, kc) = 0.25 * (RS(i, j, k) + RS(i, j, k + 1) + RS(i + 1, j, k) + RS(i + 1, j, k + 1));
        }
  } else if (nzf == nzc) {
    for (int kc = szc; kc <= ezc; ++kc)
      for (int jc = syc; jc <= eyc; ++jc)
        for (int ic = sxc; ic <= exc; ++ic) {
          const int k = kc, j = 2 * jc - 2, i = 2 * ic - 2;
          RC(ic, jc, kc) = 0.25 * (RS(i, j, k) + RS(i + 1, j, k) + RS(i, j + 1, k) + RS(i + 1, j + 1, k));
        }
  }
#undef RS
#undef RC
}

/* ----------------------------------------------------------------- mg_cor
 * mg_cor.F90:96-293: trilinear (27/9/3/1)/64 correction over coarse
 * ic = sxc-1..exc, then mg_bdry on the fine level. */
static void cor(orc_mg* m, int lC, int lF) {
  double* phif = lvl_ptr(m->work1, m, lF);
  const double* phic = lvl_ptr(m->work1, m, lC);
  const long XF = lvl_dim(m, lF, 0), YF = lvl_dim(m, lF, 1);
  const long XC = lvl_dim(m, lC, 0), YC = lvl_dim(m, lC, 1);
#define PF(i, j, k) phif[((long)(i) - 1) + XF * (((long)(j) - 1) + YF * ((long)(k) - 1))]
#define PC(i, j, k) phic[((long)(i) - 1) + XC * (((long)(j) - 1) + YC * ((long)(k) - 1))]
  const int nxc = m->nk[lC][0], nyc = m->nk[lC][1], nzc = m->nk[lC][2];
  const int nxf = m->nk[lF][0], nyf = m->nk[lF][1], nzf = m->nk[lF][2];
  const int sxc = m->sk[lC][0], exc = m->ek[lC][0];
  const int syc = m->sk[lC][1], eyc = m->ek[lC][1];
  const int szc = m->sk[lC][2], ezc = m->ek[lC][2];
  const int sxf = m->sk[lF][0], exf = m->ek[lF][0];
  const int syf = m->sk[lF][1], eyf = m->ek[lF][1];
  const int szf = m->sk[lF][2], ezf = m->ek[lF][2];
  if (nxc < nxf && nyc < nyf && nzc < nzf) {
#pragma omp parallel for schedule(static)
    for (int kc = szc - 1; kc <= ezc; ++kc) {
      const int k = 2 * kc - 1;
      for (int jc = syc - 1; jc <= eyc; ++jc) {
        const int j = 2 * jc - 1;
        for (int ic = sxc - 1; ic <= exc; ++ic) {
          const int i = 2 * ic - 1;
          const double a = PC(ic, jc, kc), b = PC(ic, jc + 1, kc), c = PC(ic, jc, kc + 1),
                       d = PC(ic, jc + 1, kc + 1), e = PC(ic + 1, jc, kc), f = PC(ic + 1, jc + 1, kc),
                       g = PC(ic + 1, jc, kc + 1), h = PC(ic + 1, jc + 1, kc + 1);
          PF(i, j, k) = PF(i, j, k) + (27.0 * a + 9.0 * b + 9.0 * c + 3.0 * d + 9.0 * e + 3.0 * f +
                                       3.0 * g + h) / 64.0;
          PF(i + 1, j, k) = PF(i + 1, j, k) + (9.0 * a + 3.0 * b + 3.0 * c + d + 27.0 * e + 9.0 * f +
                                               9.0 * g + 3.0 * h) / 64.0;
          PF(i, j + 1, k) = PF(i, j + 1, k) + (9.0 * a + 27.0 * b + 3.0 * c + 9.0 * d + 3.0 * e +
                                               9.0 * f + g + 3.0 * h) / 64.0;
          PF(i, j, k + 1) = PF(i, j, k + 1) + (9.0 * a + 3.0 * b + 27.0 * c + 9.0 * d + 3.0 * e + f +
                                               9.0 * g + 3.0 * h) / 64.0;
          PF(i + 1, j + 1, k) = PF(i + 1, j + 1, k) + (3.0 * a + 9.0 * b + c + 3.0 * d + 9.0 * e +
                                                       27.0 * f + 3.0 * g + 9.0 * h) / 64.0;
          PF(i + 1, j, k + 1) = PF(i + 1, j, k + 1) + (3.0 * a + b + 9.0 * c + 3.0 * d + 9.0 * e +
                                                       3.0 * f + 27.0 * g + 9.0 * h) / 64.0;
          PF(i, j + 1, k + 1) = PF(i, j + 1, k + 1) + (3.0 * a + 9.0 * b + 9.0 * c + 27.0 * d + e +
                                                       3.0 * f + 3.0 * g + 9.0 * h) / 64.0;
          PF(i + 1, j + 1, k + 1) = PF(i + 1, j + 1, k + 1) + (a + 3.0 * b + 3.0 * c + 9.0 * d +
                                                               3.0 * e + 9.0 * f + 9.0 * g + 27.0 * h) /
                                                                  64.0;
        }
      }
    }
  } else if (nxf == nxc && nyf == nyc) {
    for (int kc = szc - 1; kc <= ezc; ++kc) {
      const int k = 2 * kc - 1;
      for (int j = syf - 1; j <= eyf + 1; ++j)
        for (int i = sxf - 1; i <= exf + 1; ++i) {
          PF(i, j, k) = PF(i, j, k) + (3.0 * PC(i, j, kc) + PC(i, j, kc + 1)) / 4.0;
          PF(i, j, k + 1) = PF(i, j, k + 1) + (PC(i, j, kc) + 3.0 * PC(i, j, kc + 1)) / 4.0;
        }
    }
  } else if (nxf == nxc && nzf == nzc) {
    for (int k = szf - 1; k <= ezf + 1; ++k)
      for (int jc = syc - 1; jc <= eyc; ++jc) {
        const int j = 2 * jc - 1;
        for (int i = sxf - 1; i <= exf + 1; ++i) {
          PF(i, j, k) = PF(i, j, k) + (3.0 * PC(i, jc, k) + PC(i, jc + 1, k)) / 4.0;
          PF(i, j + 1, k) = PF(i, j + 1, k) + (PC(i, jc, k) + 3.0 * PC(i, jc + 1, k)) / 4.0;
        }
      }
  } else if (nyf == nyc && nzf == nzc) {
    for (int k = szf - 1; k <= ezf + 1; ++k)
      for (int j = syf - 1; j <= eyf + 1; ++j)
        for (int ic = sxc - 1; ic <= exc; ++ic) {
          const int i = 2 * ic - 1;
          PF(i, j, k) = PF(i, j, k) + (3.0 * PC(ic, j, k) + PC(ic + 1, j, k)) / 4.0;
          PF(i + 1, j, k) = PF(i + 1, j, k) + (PC(ic, j, k) + 3.0 * PC(ic + 1, j, k)) / 4.0;
        }
  } else if (nxf == nxc) {
    for (int kc = szc - 1; kc <= ezc; ++kc) {
      const int k = 2 * kc - 1;
      for (int jc = syc - 1; jc <= eyc; ++jc) {
        const int j = 2 * jc - 1;
        for (int i = sxf - 1; i <= exf + 1; ++i) {
          const double a = PC(i, jc, kc), b = PC(i, jc + 1, kc), c = PC(i, jc, kc + 1),
                       d = PC(i, jc + 1, kc + 1);
          PF(i, j, k) = PF(i, j, k) + (9.0 * a + 3.0 * b + 3.0 * c + d) / 16.0;
          PF(i, j + 1, k) = PF(i, j + 1, k) + (3.0 * a + 9.0 * b + c + 3.0 * d) / 16.0;
          PF(i, j, k + 1) = PF(i, j, k + 1) + (3.0 * a + b + 9.0 * c + 3.0 * d) / 16.0;
          PF(i, j + 1, k + 1) = PF(i, j + 1, k + 1) + (a + 3.0 * b + 3.0 * c + 9.0 * d) / 16.0;
        }
      }
    }
  } else if (nyf == nyc) {
    for (int kc = szc - 1; kc <= ezc; ++kc) {
      const int k = 2 * kc - 1;
      for (int j = syf - 1; j <= eyf + 1; ++j)
        for (int ic = sxc - 1; ic <= exc; ++ic) {
          const int i = 2 * ic - 1;
          const double a = PC(ic, j, kc), b = PC(ic + 1, j, kc), c = PC(ic, j, kc + 1),
                       d = PC(ic + 1, j, kc + 1);
          PF(i, j, k) = PF(i, j, k) + (9.0 * a + 3.0 * b + 3.0 * c + d) / 16.0;
          PF(i + 1, j, k) = PF(i + 1, j, k) + (3.0 * a + 9.0 * b + c + 3.0 * d) / 16.0;
          PF(i, j, k + 1) = PF(i, j, k + 1) + (3.0 * a + b + 9.0 * c + 3.0 * d) / 16.0;
          PF(i + 1, j, k + 1) = PF(i + 1, j, k + 1) + (a + 3.0 * b + 3.0 * c + 9.0 * d) / 16.0;
        }
    }
  } else if (nzf == nzc) {
    for (int k = szf - 1; k <= ezf + 1; ++k)
      for (int jc = syc - 1; jc <= eyc; ++jc) {
        const int j = 2 * jc - 1;
        for (int ic = sxc - 1; ic <= exc; ++ic) {
          const int i = 2 * ic - 1;
          const double a = PC(ic, jc, k), b = PC(ic + 1, jc, k), c = PC(ic, jc + 1, k),
                       d = PC(ic + 1, jc + 1, k);
          PF(i, j, k) = PF(i, j, k) + (9.0 * a + 3.0 * b + 3.0 * c + d) / 16.0;
          PF(i + 1, j, k) = PF(i + 1, j, k) + (3.0 * a + 9.0 * b + c + 3.0 * d) / 16.0;
          PF(i, j + 1, k) = PF(i, j + 1, k) + (3.0 * a + b + 9.0 * c + 3.0 * d) / 16.0;
          PF(i + 1, j + 1, k) = PF(i + 1, j + 1, k) + (a + 3.0 * b + 3.0 * c + 9.0 * d) / 16.0;
        }
      }
  }
#undef PF
#undef PC
  bdry(m, lF, phif);
}

/* --------------------------------------------------------------- mg_cycle
 * mg_cycle.F90:44-184 (RBPGS / LJ branches). */
static void cycle(orc_mg* m, double* res) {
  const int kcur = m->ngrid;
  relax(m, kcur, lvl_ptr(m->work1, m, kcur), lvl_ptr(m->work2, m, kcur), m->pre[kcur]);
  restr(m, kcur - 1, kcur, res);
  for (int kl = kcur - 1; kl >= 2; --kl) {
    relax(m, kl, lvl_ptr(m->work1, m, kl), lvl_ptr(m->work2, m, kl), m->pre[kl]);
    restr(m, kl - 1, kl, res);
  }
  relax(m, 1, lvl_ptr(m->work1, m, 1), lvl_ptr(m->work2, m, 1), m->pre[1]);
  for (int kl = 1; kl <= kcur - 1; ++kl) {
    relax(m, kl, lvl_ptr(m->work1, m, kl), lvl_ptr(m->work2, m, kl), m->post[kl]);
    cor(m, kl, kl + 1);
  }
  relax(m, kcur, lvl_ptr(m->work1, m, kcur), lvl_ptr(m->work2, m, kcur), m->post[kcur]);
}

/* ------------------------------------------------------------ mg_residual
 * mg_residual.F90:60-105 */
static double residual(orc_mg* m, double* phio, const double* phin) {
  const int l = m->ngrid;
  LVLDIMS(m, l);
  double v1 = 0.0, v2 = 0.0;
#pragma omp parallel for schedule(static) reduction(max : v1, v2)
  for (int k = m->sk[l][2]; k <= m->ek[l][2]; ++k)
    for (int j = m->sk[l][1]; j <= m->ek[l][1]; ++j)
      for (int i = m->sk[l][0]; i <= m->ek[l][0]; ++i) {
        const double an = fabs(AT(phin, i, j, k));
        const double ad = fabs(AT(phin, i, j, k) - AT(phio, i, j, k));
        v1 = v1 > an ? v1 : an;
        v2 = v2 > ad ? v2 : ad;
      }
  const double relmax = v1 > 0.0 ? v2 / v1 : 0.0;
  const long G = lvl_size(m, l);
  memcpy(phio, phin, sizeof(double) * G);
  return relmax;
}

/* ||f - A phi|| / ||f|| on the finest level with the built coefficients */
static double fine_resid_norm(orc_mg* m, const double* phi, const double* f) {
  const int l = m->ngrid;
  LVLDIMS(m, l);
  double* c[7];
  for (int q = 0; q < 7; ++q) c[q] = lvl_ptr(m->workc[q], m, l);
  double rr = 0.0, ff = 0.0;
  for (int k = m->sk[l][2]; k <= m->ek[l][2]; ++k)
    for (int j = m->sk[l][1]; j <= m->ek[l][1]; ++j)
      for (int i = m->sk[l][0]; i <= m->ek[l][0]; ++i) {
        const double ax =
            AT(c[0], i, j, k) * AT(phi, i - 1, j, k) + AT(c[1], i, j, k) * AT(phi, i + 1, j, k) +
            AT(c[2], i, j, k) * AT(phi, i, j - 1, k) + AT(c[3], i, j, k) * AT(phi, i, j + 1, k) +
            AT(c[4], i, j, k) * AT(phi, i, j, k - 1) + AT(c[5], i, j, k) * AT(phi, i, j, k + 1) +
            AT(c[6], i, j, k) * AT(phi, i, j, k);
        const double rv = AT(f, i, j, k) - ax;
        rr += rv * rv;
        ff += AT(f, i, j, k) * AT(f, i, j, k);
      }
  return ff > 0.0 ? sqrt(rr / ff) : sqrt(rr);
}

/* -------------------------------------------------------------- mg_solver
 * mg_solver.F90:71-140 */
void orc_mg_solve(orc_mg* m, double* phif, double* rhsf, int* iter, double* relmax) {
  const int ng = m->ngrid;
  build_coeffs(m);
  bdry(m, ng, phif);
  const long G = lvl_size(m, ng);
  memcpy(lvl_ptr(m->work1, m, ng), phif, sizeof(double) * G);
  memcpy(lvl_ptr(m->work2, m, ng), rhsf, sizeof(double) * G);
  double rm = 0.0;
  int it;
  if (m->stop == ANEL_STOP_RESID) {
    /* extension: stop on ||f - A phi||_2 / ||f||_2 of the fine operator;
     * the caller's rhsf is kept for the norms (work2 holds the copy the
     * cycles use) */
    const double* f = lvl_ptr(m->work2, m, ng);
    double* fsave = (double*)malloc(sizeof(double) * G);
    memcpy(fsave, f, sizeof(double) * G);
    for (it = 1; it <= m->maxcy; ++it) {
      cycle(m, rhsf);
      rm = fine_resid_norm(m, lvl_ptr(m->work1, m, ng), fsave);
      if (rm <= m->tolmax) break;
    }
    free(fsave);
    memcpy(phif, lvl_ptr(m->work1, m, ng), sizeof(double) * G);
  } else {
    for (it = 1; it <= m->maxcy; ++it) {
      cycle(m, rhsf);
      rm = residual(m, phif, lvl_ptr(m->work1, m, ng));
      if (rm <= m->tolmax) break;
    }
  }
  /* A DO loop that runs to completion leaves iter = maxcy+1 (Fortran
   * semantics), which is what the reference returns when it did not
   * converge (mg_solver.F90:114-133); the loop above does the same. */
  bdry(m, ng, phif);
  *iter = it;
  *relmax = rm;
}

void orc_mg_debug_pass(orc_mg* m, int which, double* phi, double* src) {
  const int ng = m->ngrid;
  build_coeffs(m);
  if (which == 0) {
    relax(m, ng, phi, src, 1);
  } else if (which == 1) {
    bdry(m, ng, phi);
  } else if (which == 2) {
    const long G = lvl_size(m, ng);
    double* res = (double*)calloc(G, sizeof(double));
    memcpy(lvl_ptr(m->work1, m, ng), phi, sizeof(double) * G);
    memcpy(lvl_ptr(m->work2, m, ng), src, sizeof(double) * G);
    cycle(m, res);
    memcpy(phi, lvl_ptr(m->work1, m, ng), sizeof(double) * G);
    free(res);
  }
}

void orc_mg_apply(orc_mg* m, const double* phi, double* out) {
  const int l = m->ngrid;
  LVLDIMS(m, l);
  build_coeffs(m);
  double* c[7];
  for (int q = 0; q < 7; ++q) c[q] = lvl_ptr(m->workc[q], m, l);
  for (int k = m->sk[l][2]; k <= m->ek[l][2]; ++k)
    for (int j = m->sk[l][1]; j <= m->ek[l][1]; ++j)
      for (int i = m->sk[l][0]; i <= m->ek[l][0]; ++i)
        AT(out, i, j, k) =
            AT(c[0], i, j, k) * AT(phi, i - 1, j, k) + AT(c[1], i, j, k) * AT(phi, i + 1, j, k) +
            AT(c[2], i, j, k) * AT(phi, i, j - 1, k) + AT(c[3], i, j, k) * AT(phi, i, j + 1, k) +
            AT(c[4], i, j, k) * AT(phi, i, j, k - 1) + AT(c[5], i, j, k) * AT(phi, i, j, k + 1) +
            AT(c[6], i, j, k) * AT(phi, i, j, k);
}

double orc_mg_true_resid(orc_mg* m, const double* phi, const double* f) {
  const int l = m->ngrid;
  LVLDIMS(m, l);
  const long G = lvl_size(m, l);
  double* ax = (double*)calloc(G, sizeof(double));
  orc_mg_apply(m, phi, ax);
  double rr = 0.0, ff = 0.0;
  for (int k = m->sk[l][2]; k <= m->ek[l][2]; ++k)
    for (int j = m->sk[l][1]; j <= m->ek[l][1]; ++j)
      for (int i = m->sk[l][0]; i <= m->ek[l][0]; ++i) {
        const double rv = AT(f, i, j, k) - AT(ax, i, j, k);
        rr += rv * rv;
        ff += AT(f, i, j, k) * AT(f, i, j, k);
      }
  free(ax);
  return ff > 0.0 ? sqrt(rr / ff) : sqrt(rr);
}
