/*
 * ns_oracle.c -- CPU FP64 restatement of the reference RK3 time step
 * (ANELASTIC_SL/dns/NSsolver.F90, BC.F90, Routines.F90, les/SSM.F90,
 * les/straincal.F90).  TEST INFRASTRUCTURE ONLY: used by the parity tests,
 * the smoke check and the CPU-baseline leg of bench.py; the product never
 * links or calls it.
 *
 * Serial semantics (one MPI rank, EU = EV = EW = 0, RK3CN = .true.,
 * RK3 = pcorrect = .false., LESflag = 1: Sturb.F90:110-120).  Every
 * expression follows the Fortran source left to right; compiled with
 * -ffp-contract=off.  Fortran REAL(4) literals (0.5, 0.41, 0.3) are
 * written as (double)(float) where they are not exact.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

typedef struct {
  int nx, ny, nz;
  long X, Y, Z, G;
  /* metrics, [0] = Fortran index 1 */
  const double *xe, *xc, *dxe, *dxc, *rdxe, *rdxc;
  const double *ye, *yc, *dye, *dyc, *rdye, *rdyc;
  const double *ze, *zc, *dze, *dzc, *rdze, *rdzc;
} orc_dom;

struct orc_ns {
  orc_dom d;
  anel_grid_desc g;
  anel_ns_params p;
  orc_mg* mg;
  double rRe, rPr, rSc, g_orig, gnow, time;
  int nstep;
  anel_fields f;  /* caller-owned host arrays */
  double* Ftemp;  /* RHS scratch */
  double *Csgs, *CTsgs, *CSsgs, *delg, *modS;
  double* work[4];
  double told;    /* time at the start of the last step (NSsolver.F90:272-273) */
  double* dg;     /* 16 plane-statistics profiles of Z values (orc_ns_diagnostics) */
  double *dgA, *dgB, *dgC, *dgR; /* their G-sized scratch */
};

#define IX(i, j, k) (((long)(i) - 1) + D->X * (((long)(j) - 1) + D->Y * ((long)(k) - 1)))
#define A_(a, i, j, k) (a)[IX(i, j, k)]
#define M(a, i) (a)[(i) - 1]

static const double R12 = 1.0 / 2.0; /* ratios::r_1_2 (modules.F90:203) */

/* ---------------------------------------------------------------- ghost
 * ghost() + bound_update() serial semantics (BC.F90:1-187, 334-585). */
enum { VT_U, VT_V, VT_W, VT_P, VT_RHO, VT_CFLUC, VT_PSOURCE, VT_UTEMP, VT_VTEMP, VT_WTEMP,
       VT_RTEMP, VT_S1TEMP, VT_SCAL1, VT_SCAL1TEMP };

static void vtype_info(int vt, int* l, int* rt, int* stag) {
  /* stag: 1 = u-staggered, 2 = v, 3 = w, 0 = cell centred */
  *rt = 0;
  *stag = 0;
  switch (vt) {
    case VT_U: *l = 1; *stag = 1; break;
    case VT_V: *l = 2; *stag = 2; break;
    case VT_W: *l = 3; *stag = 3; break;
    case VT_P: *l = 4; break;
    case VT_RHO: *l = 5; *rt = 1; break;
    case VT_CFLUC: *l = 6; break;
    case VT_PSOURCE: *l = 7; break;
    case VT_UTEMP: *l = 7; *stag = 1; break;
    case VT_VTEMP: *l = 7; *stag = 2; break;
    case VT_WTEMP: *l = 7; *stag = 3; break;
    case VT_RTEMP: *l = 7; break;
    case VT_S1TEMP: *l = 7; break;
    case VT_SCAL1: *l = 8; *rt = 1; break;
    default: *l = 8; break; /* VT_SCAL1TEMP */
  }
}

/* bound_update for one (dir, face) */
static void bound_update(const orc_dom* D, double* var, int btype, int face, int dir, double value,
                         int stag, int rt, int ew) {
  const int sx = 2, ex = D->nx + 1, sy = 2, ey = D->ny + 1, sz = 2, ez = D->nz + 1;
  int of1 = 0, of2 = 0;
  const double *dxt, *dyt, *dzt;
  if (stag == 1) {
    dxt = D->dxc; dyt = D->dye; dzt = D->dze; of2 = 1;
  } else if (stag == 2) {
    dxt = D->dxe; dyt = D->dyc; dzt = D->dze; of2 = 1;
  } else if (stag == 3) {
    dxt = D->dxe; dyt = D->dye; dzt = D->dzc; of2 = 1;
  } else {
    dxt = D->dxe; dyt = D->dye; dzt = D->dze; of1 = -1;
  }
  const long X = D->X, Y = D->Y, Z = D->Z;
  if (dir == 1) {
    for (long k = 1; k <= Z; ++k)
      for (long j = 1; j <= Y; ++j) {
        double* L = &A_(var, 1, j, k);
        /* L[i-1] = var(i,j,k) */
        if (btype == 1) {
          if (face == 1) L[sx - 2] = value;
          else L[ex] = value;
        } else if (btype == 2) {
          if (face == 1) {
            if (rt == 1) L[sx - 1] = L[sx] - value * M(dxt, sx + 1 + of1);
            L[sx - 2] = L[sx - 1] - value * M(dxt, sx + of1);
          } else {
            if (rt == 1) L[ex - 1] = L[ex - 2] + value * M(dxt, ex - 1 + of2);
            L[ex] = L[ex - 1] + value * M(dxt, ex + of2);
          }
        } else if (btype == 3) {
          L[sx - 2] = L[ex - 1];
          L[ex] = L[sx - 1];
        } else if (btype == 4) {
          if (face == 1) L[sx - 2] = L[sx - 1] - value * M(dxt, sx + of1);
          else L[ex] = L[ex - 1] + value * M(dxt, ex + of2);
        } else if (btype == 8) {
          if (face == 1) L[sx - 2] = 2.0 * L[sx - 1] - L[sx];
          else L[ex] = 2.0 * L[ex - 1] - L[ex - 2];
        }
      }
  } else if (dir == 2) {
    for (long k = 1; k <= Z; ++k)
      for (long i = 1; i <= X; ++i) {
#define V2(j) A_(var, i, j, k)
        if (btype == 1) {
          if (face == 1) V2(sy - 1) = value;
          else V2(ey + 1) = value;
        } else if (btype == 2) {
          if (face == 1) {
            if (rt == 1) V2(sy) = V2(sy + 1) - value * M(dyt, sy + 1 + of1);
            V2(sy - 1) = V2(sy) - value * M(dyt, sy + of1);
          } else {
            if (rt == 1) V2(ey) = V2(ey - 1) + value * M(dyt, ey - 1 + of2);
            V2(ey + 1) = V2(ey) + value * M(dyt, ey + of2);
          }
        } else if (btype == 3) {
          V2(sy - 1) = V2(ey);
          V2(ey + 1) = V2(sy);
        } else if (btype == 4) {
          if (face == 1) V2(sy - 1) = V2(sy) - value * M(dyt, sy + of1);
          else V2(ey + 1) = V2(ey) + value * M(dyt, ey + of2);
        }
#undef V2
      }
  } else {
    const int iW = (stag == 3) ? ew : 0;
    for (long j = 1; j <= Y; ++j)
      for (long i = 1; i <= X; ++i) {
#define V3(k) A_(var, i, j, k)
        if (btype == 1) {
          if (face == 1) V3(sz - 1) = value;
          else V3(ez + 1 - iW) = value;
        } else if (btype == 2) {
          if (face == 1) {
            if (rt == 1) V3(sz) = V3(sz + 1) - value * M(dzt, sz + 1 + of1);
            V3(sz - 1) = V3(sz) - value * M(dzt, sz + of1);
          } else {
            if (rt == 1) V3(ez - iW) = V3(ez - 1 - iW) + value * M(dzt, ez - 1 + of2 - iW);
            V3(ez + 1 - iW) = V3(ez - iW) + value * M(dzt, ez + of2 - iW);
          }
        } else if (btype == 3) {
          V3(sz - 1) = V3(ez - iW);
          V3(ez + 1 - iW) = V3(sz);
        } else if (btype == 4) {
          if (face == 1) V3(sz - 1) = V3(sz) - value * M(dzt, sz + of1);
          else V3(ez + 1 - iW) = V3(ez - iW) + value * M(dzt, ez + of2 - iW);
        } else if (btype == 6) {
          if (face == 1) V3(sz - 1) = 2.0 * value - 1.0 * V3(sz);
          else V3(ez + 1 - iW) = 2.0 * value - 1.0 * V3(ez - iW);
        } else if (btype == 7) {
          if (face == 1) {
            V3(sz) = 0.0;
            V3(sz - 1) = -1.0 * V3(sz + 1);
          } else {
            V3(ez) = 0.0;
            V3(ez + 1 - iW) = -1.0 * V3(ez - iW - 1);
          }
        }
        /* SET EXTRA POINT TO ZERO (BC.F90:526-527) */
        if (face == 2 && iW == 1) V3(ez + 1) = 0.0;
#undef V3
      }
  }
}

static void ghost(const orc_ns* s, double* var, int vt) {
  const orc_dom* D = &s->d;
  const long X = D->X, Y = D->Y, Z = D->Z;
  const int sx = 2, ex = D->nx + 1, sy = 2, ey = D->ny + 1, sz = 2, ez = D->nz + 1;
  /* full periodic wrap (BC.F90:55-66) */
  for (long k = 1; k <= Z; ++k)
    for (long j = 1; j <= Y; ++j) {
      A_(var, sx - 1, j, k) = A_(var, ex, j, k);
      A_(var, ex + 1, j, k) = A_(var, sx, j, k);
    }
  for (long k = 1; k <= Z; ++k)
    for (long i = 1; i <= X; ++i) {
      A_(var, i, sy - 1, k) = A_(var, i, ey, k);
      A_(var, i, ey + 1, k) = A_(var, i, sy, k);
    }
  for (long j = 1; j <= Y; ++j)
    for (long i = 1; i <= X; ++i) {
      A_(var, i, j, sz - 1) = A_(var, i, j, ez);
      A_(var, i, j, ez + 1) = A_(var, i, j, sz);
    }
  int l, rt, stag;
  vtype_info(vt, &l, &rt, &stag);
  for (int n = 1; n <= 3; ++n)
    for (int m = 1; m <= 2; ++m) {
      const int tb = s->p.tb[n - 1][m - 1][l - 1];
      const int tb1 = s->p.tb[n - 1][0][l - 1];
      if (tb1 != 3 || m == 1)
        bound_update(D, var, tb, m, n, s->p.vb[n - 1][m - 1][l - 1], stag, rt, s->p.ew);
    }
}

/* ------------------------------------------------------------ create */
orc_ns* orc_ns_create(const anel_grid_desc* g, const anel_mg_params* mgp, const anel_ns_params* np,
                      int* stat) {
  orc_ns* s = (orc_ns*)calloc(1, sizeof(orc_ns));
  s->g = *g;
  s->p = *np;
  orc_dom* D = &s->d;
  D->nx = g->nx;
  D->ny = g->ny;
  D->nz = g->nz;
  D->X = g->nx + 2;
  D->Y = g->ny + 2;
  D->Z = g->nz + 2;
  D->G = D->X * D->Y * D->Z;
  D->xe = g->xe; D->xc = g->xc; D->dxe = g->dxe; D->dxc = g->dxc; D->rdxe = g->rdxe; D->rdxc = g->rdxc;
  D->ye = g->ye; D->yc = g->yc; D->dye = g->dye; D->dyc = g->dyc; D->rdye = g->rdye; D->rdyc = g->rdyc;
  D->ze = g->ze; D->zc = g->zc; D->dze = g->dze; D->dzc = g->dzc; D->rdze = g->rdze; D->rdzc = g->rdzc;
  s->rRe = 1.0 / np->Re;
  s->rPr = 1.0 / np->Pr;
  s->rSc = 1.0 / np->Sc;
  s->g_orig = np->g_final;
  s->gnow = np->g_init;
  s->mg = orc_mg_create(g, mgp, stat);
  if (*stat != 0) return s;
  s->Ftemp = (double*)calloc(D->G, sizeof(double));
  s->Csgs = (double*)calloc(D->G, sizeof(double));
  s->CTsgs = (double*)calloc(D->G, sizeof(double));
  s->CSsgs = (double*)calloc(D->G, sizeof(double));
  s->delg = (double*)calloc(D->G, sizeof(double));
  s->modS = (double*)calloc(D->G, sizeof(double));
  for (int q = 0; q < 4; ++q) s->work[q] = (double*)calloc(D->G, sizeof(double));
  s->nstep = 1;
  s->told = 1.0e-16; /* NSsolver.F90:47 */
  return s;
}

void orc_ns_destroy(orc_ns* s) {
  if (!s) return;
  orc_mg_destroy(s->mg);
  free(s->Ftemp);
  free(s->Csgs);
  free(s->CTsgs);
  free(s->CSsgs);
  free(s->delg);
  free(s->modS);
  for (int q = 0; q < 4; ++q) free(s->work[q]);
  free(s->dg);
  free(s->dgA);
  free(s->dgB);
  free(s->dgC);
  free(s->dgR);
  free(s);
}

void orc_ns_bind(orc_ns* s, const anel_fields* f) { s->f = *f; }
void orc_ns_set_clock(orc_ns* s, double time, int nstep) {
  s->time = time;
  s->nstep = nstep;
}

static int les_on(const orc_ns* s) {
  return s->p.vmodel != ANEL_MODEL_DNS;
}

/* ---------------------------------------------------------------- u1_rhs
 * NSsolver.F90:585-860 (DNS linear + non-linear, SSM LES terms). */
static void u1_rhs(orc_ns* s, double* Ut) {
  const orc_dom* D = &s->d;
  const double *un = s->f.u, *vn = s->f.v, *wn = s->f.w, *r = s->f.r, *nuT = s->f.nuT;
  const double rRe = s->rRe;
  memset(Ut, 0, sizeof(double) * D->G);
  const int sx = 2, ex = D->nx + 1, sy = 2, ey = D->ny + 1, sz = 2, ez = D->nz + 1;
  #pragma omp parallel for schedule(static)
  for (int k = sz; k <= ez; ++k)
    for (int j = sy; j <= ey; ++j)
      for (int i = sx; i <= ex; ++i)
        A_(Ut, i, j, k) = A_(Ut, i, j, k) +
                          rRe * ((A_(un, i + 1, j, k) - A_(un, i, j, k)) * M(D->rdxc, i + 1) -
                                 (A_(un, i, j, k) - A_(un, i - 1, j, k)) * M(D->rdxc, i)) *
                              M(D->rdxe, i) +
                          rRe * ((A_(un, i, j + 1, k) - A_(un, i, j, k)) * M(D->rdye, j) -
                                 (A_(un, i, j, k) - A_(un, i, j - 1, k)) * M(D->rdye, j - 1)) *
                              M(D->rdyc, j);
  #pragma omp parallel for schedule(static)
  for (int k = sz; k <= ez; ++k)
    for (int j = sy; j <= ey; ++j)
      for (int i = sx; i <= ex; ++i) {
        double ua2 = R12 * (A_(un, i + 1, j, k) + A_(un, i, j, k));
        double ua1 = R12 * (A_(un, i, j, k) + A_(un, i - 1, j, k));
        A_(Ut, i, j, k) = A_(Ut, i, j, k) + (ua1 * ua1 - ua2 * ua2) * M(D->rdxe, i);
        ua2 = R12 * (A_(un, i, j, k + 1) + A_(un, i, j, k));
        ua1 = R12 * (A_(un, i, j, k) + A_(un, i, j, k - 1));
        const double ra2 = R12 * (A_(r, i, j, k + 1) + A_(r, i, j, k));
        const double ra1 = R12 * (A_(r, i, j, k) + A_(r, i, j, k - 1));
        const double wa2 = R12 * (A_(wn, i + 1, j, k) + A_(wn, i, j, k));
        const double wa1 = R12 * (A_(wn, i + 1, j, k - 1) + A_(wn, i, j, k - 1));
        A_(Ut, i, j, k) =
            A_(Ut, i, j, k) + (ra1 * ua1 * wa1 - ra2 * ua2 * wa2) * M(D->rdzc, k) / A_(r, i, j, k);
        ua2 = R12 * (A_(un, i, j + 1, k) + A_(un, i, j, k));
        ua1 = R12 * (A_(un, i, j, k) + A_(un, i, j - 1, k));
        const double va2 = R12 * (A_(vn, i + 1, j, k) + A_(vn, i, j, k));
        const double va1 = R12 * (A_(vn, i + 1, j - 1, k) + A_(vn, i, j - 1, k));
        A_(Ut, i, j, k) = A_(Ut, i, j, k) + (ua1 * va1 - ua2 * va2) * M(D->rdyc, j);
      }
  if (les_on(s)) {
    #pragma omp parallel for schedule(static)
    for (int k = sz; k <= ez; ++k)
      for (int j = sy; j <= ey; ++j)
        for (int i = sx; i <= ex; ++i) {
          A_(Ut, i, j, k) =
              A_(Ut, i, j, k) -
              1 * 2.0 *
                  (A_(nuT, i + 1, j, k) * (A_(un, i + 1, j, k) - A_(un, i, j, k)) * M(D->rdxc, i + 1) -
                   A_(nuT, i, j, k) * (A_(un, i, j, k) - A_(un, i - 1, j, k)) * M(D->rdxc, i)) *
                  M(D->rdxe, i);
          double n1 = 0.25 * (A_(nuT, i, j, k) + A_(nuT, i + 1, j, k) + A_(nuT, i, j - 1, k) +
                              A_(nuT, i + 1, j - 1, k));
          double n2 = 0.25 * (A_(nuT, i, j, k) + A_(nuT, i + 1, j, k) + A_(nuT, i, j + 1, k) +
                              A_(nuT, i + 1, j + 1, k));
          A_(Ut, i, j, k) = A_(Ut, i, j, k) -
                            1 * 1.0 *
                                (n2 * (A_(un, i, j + 1, k) - A_(un, i, j, k)) * M(D->rdye, j) -
                                 n1 * (A_(un, i, j, k) - A_(un, i, j - 1, k)) * M(D->rdye, j - 1)) *
                                M(D->rdyc, j);
          A_(Ut, i, j, k) = A_(Ut, i, j, k) -
                            1 * 1.0 *
                                (n2 * (A_(vn, i + 1, j + 1, k) - A_(vn, i, j + 1, k)) * M(D->rdxe, i) -
                                 n1 * (A_(vn, i + 1, j, k) - A_(vn, i, j, k)) * M(D->rdxe, i)) *
                                M(D->rdyc, j);
          n1 = 0.25 * (A_(nuT, i, j, k) + A_(nuT, i + 1, j, k) + A_(nuT, i, j, k - 1) +
                       A_(nuT, i + 1, j, k - 1));
          n2 = 0.25 * (A_(nuT, i, j, k) + A_(nuT, i + 1, j, k) + A_(nuT, i, j, k + 1) +
                       A_(nuT, i + 1, j, k + 1));
          const double ra2 = R12 * (A_(r, i, j, k + 1) + A_(r, i, j, k));
          const double ra1 = R12 * (A_(r, i, j, k) + A_(r, i, j, k - 1));
          A_(Ut, i, j, k) =
              A_(Ut, i, j, k) -
              1 * 1.0 *
                  (ra2 * n2 * (A_(wn, i + 1, j, k) - A_(wn, i, j, k)) * M(D->rdxe, i) -
                   ra1 * n1 * (A_(wn, i + 1, j, k - 1) - A_(wn, i, j, k - 1)) * M(D->rdxe, i)) *
                  M(D->rdzc, k) / A_(r, i, j, k);
        }
  }
  ghost(s, Ut, VT_UTEMP);
}

/* ---------------------------------------------------------------- u2_rhs
 * NSsolver.F90:863-1136 */
static void u2_rhs(orc_ns* s, double* Vt) {
  const orc_dom* D = &s->d;
  const double *un = s->f.u, *vn = s->f.v, *wn = s->f.w, *r = s->f.r, *nuT = s->f.nuT;
  const double rRe = s->rRe;
  memset(Vt, 0, sizeof(double) * D->G);
  const int sx = 2, ex = D->nx + 1, sy = 2, ey = D->ny + 1, sz = 2, ez = D->nz + 1;
  #pragma omp parallel for schedule(static)
  for (int k = sz; k <= ez; ++k)
    for (int j = sy; j <= ey; ++j)
      for (int i = sx; i <= ex; ++i)
        A_(Vt, i, j, k) = A_(Vt, i, j, k) +
                          rRe * ((A_(vn, i + 1, j, k) - A_(vn, i, j, k)) * M(D->rdxe, i) -
                                 (A_(vn, i, j, k) - A_(vn, i - 1, j, k)) * M(D->rdxe, i - 1)) *
                              M(D->rdxc, i) +
                          rRe * ((A_(vn, i, j + 1, k) - A_(vn, i, j, k)) * M(D->rdyc, j + 1) -
                                 (A_(vn, i, j, k) - A_(vn, i, j - 1, k)) * M(D->rdyc, j)) *
                              M(D->rdye, j);
  #pragma omp parallel for schedule(static)
  for (int k = sz; k <= ez; ++k)
    for (int j = sy; j <= ey; ++j)
      for (int i = sx; i <= ex; ++i) {
        double va1 = 0.5 * (A_(vn, i, j + 1, k) + A_(vn, i, j, k));
        double va2 = 0.5 * (A_(vn, i, j, k) + A_(vn, i, j - 1, k));
        A_(Vt, i, j, k) = A_(Vt, i, j, k) - (va1 * va1 - va2 * va2) * M(D->rdye, j);
        va1 = 0.5 * (A_(vn, i + 1, j, k) + A_(vn, i, j, k));
        va2 = 0.5 * (A_(vn, i, j, k) + A_(vn, i - 1, j, k));
        const double ua1 = 0.5 * (A_(un, i, j + 1, k) + A_(un, i, j, k));
        const double ua2 = 0.5 * (A_(un, i - 1, j + 1, k) + A_(un, i - 1, j, k));
        A_(Vt, i, j, k) = A_(Vt, i, j, k) - (ua1 * va1 - ua2 * va2) * M(D->rdxc, i);
        va1 = 0.5 * (A_(vn, i, j, k + 1) + A_(vn, i, j, k));
        va2 = 0.5 * (A_(vn, i, j, k) + A_(vn, i, j, k - 1));
        const double ra1 = 0.5 * (A_(r, i, j, k + 1) + A_(r, i, j, k));
        const double ra2 = 0.5 * (A_(r, i, j, k) + A_(r, i, j, k - 1));
        const double wa1 = 0.5 * (A_(wn, i, j + 1, k) + A_(wn, i, j, k));
        const double wa2 = 0.5 * (A_(wn, i, j + 1, k - 1) + A_(wn, i, j, k - 1));
        A_(Vt, i, j, k) =
            A_(Vt, i, j, k) - (ra1 * wa1 * va1 - ra2 * wa2 * va2) * M(D->rdzc, k) / A_(r, i, j, k);
      }
  if (les_on(s)) {
    #pragma omp parallel for schedule(static)
    for (int k = sz; k <= ez; ++k)
      for (int j = sy; j <= ey; ++j)
        for (int i = sx; i <= ex; ++i) {
          double n1 = 0.25 * (A_(nuT, i, j, k) + A_(nuT, i - 1, j, k) + A_(nuT, i, j + 1, k) +
                              A_(nuT, i - 1, j + 1, k));
          double n2 = 0.25 * (A_(nuT, i, j, k) + A_(nuT, i + 1, j, k) + A_(nuT, i, j + 1, k) +
                              A_(nuT, i + 1, j + 1, k));
          A_(Vt, i, j, k) = A_(Vt, i, j, k) -
                            1 * 1.0 *
                                (n2 * (A_(vn, i + 1, j, k) - A_(vn, i, j, k)) * M(D->rdxe, i) -
                                 n1 * (A_(vn, i, j, k) - A_(vn, i - 1, j, k)) * M(D->rdxe, i - 1)) *
                                M(D->rdxc, i);
          A_(Vt, i, j, k) = A_(Vt, i, j, k) -
                            1 * 1.0 *
                                (n2 * (A_(un, i + 1, j + 1, k) - A_(un, i + 1, j, k)) * M(D->rdye, j) -
                                 n1 * (A_(un, i, j + 1, k) - A_(un, i, j, k)) * M(D->rdye, j)) *
                                M(D->rdxc, i);
          A_(Vt, i, j, k) =
              A_(Vt, i, j, k) -
              1 * 2.0 *
                  (A_(nuT, i, j + 1, k) * (A_(vn, i, j + 1, k) - A_(vn, i, j, k)) * M(D->rdyc, j + 1) -
                   A_(nuT, i, j, k) * (A_(vn, i, j, k) - A_(vn, i, j - 1, k)) * M(D->rdyc, j)) *
                  M(D->rdye, j);
          n1 = 0.25 * (A_(nuT, i, j, k) + A_(nuT, i, j + 1, k) + A_(nuT, i, j, k - 1) +
                       A_(nuT, i, j + 1, k - 1));
          n2 = 0.25 * (A_(nuT, i, j, k) + A_(nuT, i, j + 1, k) + A_(nuT, i, j, k + 1) +
                       A_(nuT, i, j + 1, k + 1));
          const double ra1 = 0.5 * (A_(r, i, j, k + 1) + A_(r, i, j, k));
          const double ra2 = 0.5 * (A_(r, i, j, k) + A_(r, i, j, k - 1));
          /* the reference pairs raver2 (lower face) with nuTaver2 (upper) */
          A_(Vt, i, j, k) =
              A_(Vt, i, j, k) -
              1 * 1.0 *
                  (ra2 * n2 * (A_(wn, i, j + 1, k) - A_(wn, i, j, k)) * M(D->rdye, j) -
                   ra1 * n1 * (A_(wn, i, j + 1, k - 1) - A_(wn, i, j, k - 1)) * M(D->rdye, j)) *
                  M(D->rdzc, k) / A_(r, i, j, k);
        }
  }
  ghost(s, Vt, VT_VTEMP);
}

/* ---------------------------------------------------------------- u3_rhs
 * NSsolver.F90:1138-1432 (density_mean at :1201 is dead: its result is
 * not used). */
static void u3_rhs(orc_ns* s, double* Wt) {
  const orc_dom* D = &s->d;
  const double *un = s->f.u, *vn = s->f.v, *wn = s->f.w, *r = s->f.r, *nuT = s->f.nuT;
  const double *rhon = s->f.rho, *bg = s->f.densityBG;
  const double rRe = s->rRe, g = s->gnow;
  memset(Wt, 0, sizeof(double) * D->G);
  const int sx = 2, ex = D->nx + 1, sy = 2, ey = D->ny + 1, sz = 2, ez = D->nz + 1;
  const int kend = ez - s->p.ew; /* k = sz..ez-EW */
  #pragma omp parallel for schedule(static)
  for (int k = sz; k <= kend; ++k)
    for (int j = sy; j <= ey; ++j)
      for (int i = sx; i <= ex; ++i)
        A_(Wt, i, j, k) = A_(Wt, i, j, k) +
                          R12 * g *
                              ((A_(rhon, i, j, k + 1) - A_(bg, i, j, k + 1)) +
                               (A_(rhon, i, j, k) - A_(bg, i, j, k))) /
                              (R12 * (A_(bg, i, j, k + 1) + A_(bg, i, j, k)));
  #pragma omp parallel for schedule(static)
  for (int k = sz; k <= kend; ++k)
    for (int j = sy; j <= ey; ++j)
      for (int i = sx; i <= ex; ++i)
        A_(Wt, i, j, k) = A_(Wt, i, j, k) +
                          rRe * ((A_(wn, i + 1, j, k) - A_(wn, i, j, k)) * M(D->rdxe, i) -
                                 (A_(wn, i, j, k) - A_(wn, i - 1, j, k)) * M(D->rdxe, i - 1)) *
                              M(D->rdxc, i) +
                          rRe * ((A_(wn, i, j + 1, k) - A_(wn, i, j, k)) * M(D->rdye, j) -
                                 (A_(wn, i, j, k) - A_(wn, i, j - 1, k)) * M(D->rdye, j - 1)) *
                              M(D->rdyc, j);
  #pragma omp parallel for schedule(static)
  for (int k = sz; k <= kend; ++k)
    for (int j = sy; j <= ey; ++j)
      for (int i = sx; i <= ex; ++i) {
        double wa1 = 0.5 * (A_(wn, i, j, k + 1) + A_(wn, i, j, k));
        double wa2 = 0.5 * (A_(wn, i, j, k) + A_(wn, i, j, k - 1));
        A_(Wt, i, j, k) = A_(Wt, i, j, k) -
                          (A_(r, i, j, k) * wa1 * wa1 - A_(r, i, j, k + 1) * wa2 * wa2) * M(D->rdze, k) /
                              (0.5 * (A_(r, i, j, k) + A_(r, i, j, k + 1)));
        wa1 = 0.5 * (A_(wn, i + 1, j, k) + A_(wn, i, j, k));
        wa2 = 0.5 * (A_(wn, i, j, k) + A_(wn, i - 1, j, k));
        const double ua1 = 0.5 * (A_(un, i, j, k + 1) + A_(un, i, j, k));
        const double ua2 = 0.5 * (A_(un, i - 1, j, k + 1) + A_(un, i - 1, j, k));
        A_(Wt, i, j, k) = A_(Wt, i, j, k) - (ua1 * wa1 - ua2 * wa2) * M(D->rdxc, i);
        wa1 = 0.5 * (A_(wn, i, j + 1, k) + A_(wn, i, j, k));
        wa2 = 0.5 * (A_(wn, i, j, k) + A_(wn, i, j - 1, k));
        const double va1 = 0.5 * (A_(vn, i, j, k + 1) + A_(vn, i, j, k));
        const double va2 = 0.5 * (A_(vn, i, j - 1, k + 1) + A_(vn, i, j - 1, k));
        A_(Wt, i, j, k) = A_(Wt, i, j, k) - (va1 * wa1 - va2 * wa2) * M(D->rdyc, j);
      }
  if (les_on(s)) {
    #pragma omp parallel for schedule(static)
    for (int k = sz; k <= kend; ++k)
      for (int j = sy; j <= ey; ++j)
        for (int i = sx; i <= ex; ++i) {
          double n1 = 0.25 * (A_(nuT, i, j, k) + A_(nuT, i - 1, j, k) + A_(nuT, i, j, k + 1) +
                              A_(nuT, i - 1, j, k + 1));
          double n2 = 0.25 * (A_(nuT, i, j, k) + A_(nuT, i + 1, j, k) + A_(nuT, i, j, k + 1) +
                              A_(nuT, i + 1, j, k + 1));
          A_(Wt, i, j, k) = A_(Wt, i, j, k) -
                            1 * 1.0 *
                                (n2 * (A_(wn, i + 1, j, k) - A_(wn, i, j, k)) * M(D->rdxe, i) -
                                 n1 * (A_(wn, i, j, k) - A_(wn, i - 1, j, k)) * M(D->rdxe, i - 1)) *
                                M(D->rdxc, i);
          A_(Wt, i, j, k) = A_(Wt, i, j, k) -
                            1 * 1.0 *
                                (n2 * (A_(un, i + 1, j, k + 1) - A_(un, i + 1, j, k)) * M(D->rdze, k) -
                                 n1 * (A_(un, i, j, k + 1) - A_(un, i, j, k)) * M(D->rdze, k)) *
                                M(D->rdxc, i);
          n1 = 0.25 * (A_(nuT, i, j, k) + A_(nuT, i, j - 1, k) + A_(nuT, i, j, k + 1) +
                       A_(nuT, i, j - 1, k + 1));
          n2 = 0.25 * (A_(nuT, i, j, k) + A_(nuT, i, j + 1, k) + A_(nuT, i, j, k + 1) +
                       A_(nuT, i, j + 1, k + 1));
          A_(Wt, i, j, k) = A_(Wt, i, j, k) -
                            1 * 1.0 *
                                (n2 * (A_(wn, i, j + 1, k) - A_(wn, i, j, k)) * M(D->rdye, j) -
                                 n1 * (A_(wn, i, j, k) - A_(wn, i, j - 1, k)) * M(D->rdye, j - 1)) *
                                M(D->rdyc, j);
          A_(Wt, i, j, k) = A_(Wt, i, j, k) -
                            1 * 1.0 *
                                (n2 * (A_(vn, i, j + 1, k + 1) - A_(vn, i, j + 1, k)) * M(D->rdze, k) -
                                 n1 * (A_(vn, i, j, k + 1) - A_(vn, i, j, k)) * M(D->rdze, k)) *
                                M(D->rdyc, j);
        }
  }
  ghost(s, Wt, VT_WTEMP);
}

/* ------------------------------------------------ rho_rhs / scal1_rhs
 * NSsolver.F90:1667-1838 and 1841-2020.  The scalar LES term keeps the
 * reference's sign slip nappaT(i)-nappaT(i-1) in the lower-face average
 * (:1970,1975). */
static void scalar_rhs(orc_ns* s, double* St, int is_rho) {
  const orc_dom* D = &s->d;
  const double *un = s->f.u, *vn = s->f.v, *wn = s->f.w, *r = s->f.r;
  const double* c = is_rho ? s->f.rho : s->f.scal1;
  const double* kT = is_rho ? s->f.kappaT : s->f.nappaT;
  const double Dk = is_rho ? s->rRe * s->rPr : s->rRe * s->rSc;
  const int model = is_rho ? s->p.rmodel : s->p.smodel;
  memset(St, 0, sizeof(double) * D->G);
  const int sx = 2, ex = D->nx + 1, sy = 2, ey = D->ny + 1, sz = 2, ez = D->nz + 1;
  #pragma omp parallel for schedule(static)
  for (int k = sz; k <= ez; ++k)
    for (int j = sy; j <= ey; ++j)
      for (int i = sx; i <= ex; ++i)
        A_(St, i, j, k) = A_(St, i, j, k) +
                          Dk * ((A_(c, i + 1, j, k) - A_(c, i, j, k)) * M(D->rdxe, i) -
                                (A_(c, i, j, k) - A_(c, i - 1, j, k)) * M(D->rdxe, i - 1)) *
                              M(D->rdxc, i) +
                          Dk * ((A_(c, i, j + 1, k) - A_(c, i, j, k)) * M(D->rdye, j) -
                                (A_(c, i, j, k) - A_(c, i, j - 1, k)) * M(D->rdye, j - 1)) *
                              M(D->rdyc, j);
  #pragma omp parallel for schedule(static)
  for (int k = sz; k <= ez; ++k)
    for (int j = sy; j <= ey; ++j)
      for (int i = sx; i <= ex; ++i) {
        double c2 = 0.5 * (A_(c, i + 1, j, k) + A_(c, i, j, k));
        double c1 = 0.5 * (A_(c, i, j, k) + A_(c, i - 1, j, k));
        A_(St, i, j, k) =
            A_(St, i, j, k) + (A_(un, i - 1, j, k) * c1 - A_(un, i, j, k) * c2) * M(D->rdxc, i);
        c2 = 0.5 * (A_(c, i, j + 1, k) + A_(c, i, j, k));
        c1 = 0.5 * (A_(c, i, j, k) + A_(c, i, j - 1, k));
        A_(St, i, j, k) =
            A_(St, i, j, k) + (A_(vn, i, j - 1, k) * c1 - A_(vn, i, j, k) * c2) * M(D->rdyc, j);
        c2 = 0.5 * (A_(c, i, j, k + 1) + A_(c, i, j, k));
        c1 = 0.5 * (A_(c, i, j, k) + A_(c, i, j, k - 1));
        if (is_rho) {
          const double ra2 = 0.5 * (A_(r, i, j, k + 1) + A_(r, i, j, k));
          const double ra1 = 0.5 * (A_(r, i, j, k) + A_(r, i, j, k - 1));
          A_(St, i, j, k) = A_(St, i, j, k) + (ra1 * A_(wn, i, j, k - 1) * c1 -
                                               ra2 * A_(wn, i, j, k) * c2) *
                                                  M(D->rdzc, k) / A_(r, i, j, k);
        } else {
          A_(St, i, j, k) =
              A_(St, i, j, k) + (A_(wn, i, j, k - 1) * c1 - A_(wn, i, j, k) * c2) * M(D->rdzc, k);
        }
      }
  if (model != ANEL_MODEL_DNS) {
    #pragma omp parallel for schedule(static)
    for (int k = sz; k <= ez; ++k)
      for (int j = sy; j <= ey; ++j)
        for (int i = sx; i <= ex; ++i) {
          double k2 = 0.5 * (A_(kT, i + 1, j, k) + A_(kT, i, j, k));
          double k1 = is_rho ? 0.5 * (A_(kT, i, j, k) + A_(kT, i - 1, j, k))
                             : 0.5 * (A_(kT, i, j, k) - A_(kT, i - 1, j, k));
          A_(St, i, j, k) = A_(St, i, j, k) -
                            1 * 1.0 *
                                (k2 * (A_(c, i + 1, j, k) - A_(c, i, j, k)) * M(D->rdxe, i) -
                                 k1 * (A_(c, i, j, k) - A_(c, i - 1, j, k)) * M(D->rdxe, i - 1)) *
                                M(D->rdxc, i);
          k2 = 0.5 * (A_(kT, i, j + 1, k) + A_(kT, i, j, k));
          k1 = is_rho ? 0.5 * (A_(kT, i, j, k) + A_(kT, i, j - 1, k))
                      : 0.5 * (A_(kT, i, j, k) - A_(kT, i, j - 1, k));
          A_(St, i, j, k) = A_(St, i, j, k) -
                            1 * 1.0 *
                                (k2 * (A_(c, i, j + 1, k) - A_(c, i, j, k)) * M(D->rdye, j) -
                                 k1 * (A_(c, i, j, k) - A_(c, i, j - 1, k)) * M(D->rdye, j - 1)) *
                                M(D->rdyc, j);
        }
  }
  ghost(s, St, is_rho ? VT_RTEMP : VT_SCAL1TEMP);
}

/* var_advance (NSsolver.F90:2225-2264), interior only */
static void var_advance(const orc_ns* s, const double* v1, double* v2, double f1, double f2, double f3) {
  const orc_dom* D = &s->d;
  #pragma omp parallel for schedule(static)
  for (int k = 2; k <= D->nz + 1; ++k)
    for (int j = 2; j <= D->ny + 1; ++j)
      for (int i = 2; i <= D->nx + 1; ++i)
        A_(v2, i, j, k) = f1 * A_(v2, i, j, k) + f2 * A_(v1, i, j, k) * f3;
}

/* Thomas of mg_relax.F90:541-595 (a, b overwritten, c untouched) */
static void thomas_ns(double* a, double* b, const double* c, double* G, int n) {
  for (int j = 1; j <= n - 1; ++j) {
    a[j] = -a[j] / b[j - 1];
    b[j] = b[j] + a[j] * c[j - 1];
    G[j] = G[j] + a[j] * G[j - 1];
  }
  G[n - 1] = G[n - 1] / b[n - 1];
  for (int j = n - 1; j >= 1; --j) G[j - 1] = (G[j - 1] - c[j - 1] * G[j]) / b[j - 1];
}

/* -------------------------------------------------- var_advance_CN_PL
 * NSsolver.F90:3054-3465 with f1 = 1, f3 = 1 (as rk_ss calls it),
 * Deddy = 0 (:3116), pcorrect = .false..  var: 1 u, 2 v, 3 w, 5 rho,
 * 8 scal1.  The sub/sup/diag/rhs arrays are built over the ghosted (i,j)
 * range, ghosted as 'cfluc', given the wall rows, then solved by Thomas
 * over k = 1..nz+2 per interior column. */
static void cn_pl(orc_ns* s, const double* q, double* u, double a3, double rkdt, int var) {
  const orc_dom* D = &s->d;
  const double* r = s->f.r;
  const double rRe = s->rRe;
  double *sub = s->work[0], *diag = s->work[1], *sup = s->work[2], *rhs = s->work[3];
  const long G = D->G;
  memset(sub, 0, sizeof(double) * G);
  memset(sup, 0, sizeof(double) * G);
  memset(diag, 0, sizeof(double) * G);
  memset(rhs, 0, sizeof(double) * G);
  const int sz = 2, ez = D->nz + 1;
  const double H = (double)(float)0.5; /* REAL(4) literal 0.5 (exact) */
  const int les = les_on(s);
  const double* kT = (var == 5) ? s->f.kappaT : (var == 8) ? s->f.nappaT : s->f.nuT;
  /* the LES block of var_advance_CN_PL is gated on Vmodel for every
   * variable, scalars included (NSsolver.F90:3160-3190) */
  const int les_var = les;
#pragma omp parallel for schedule(static)
  for (long j = 1; j <= D->Y; ++j)
    for (long i = 1; i <= D->X; ++i) {
      if (var != 3) {
        for (int k = sz; k <= ez; ++k) {
          double t1, t2;
          const double ra1 = H * (A_(r, i, j, k + 1) + A_(r, i, j, k));
          const double ra2 = H * (A_(r, i, j, k) + A_(r, i, j, k - 1));
          if (var == 1 || var == 2) {
            t1 = (rRe + 0.0) * ra1 / A_(r, i, j, k);
            t2 = (rRe + 0.0) * ra2 / A_(r, i, j, k);
          } else if (var == 5) {
            t1 = (rRe * s->rPr + 0.0) * ra1 / A_(r, i, j, k);
            t2 = (rRe * s->rPr + 0.0) * ra2 / A_(r, i, j, k);
          } else {
            t1 = rRe * s->rSc + 0.0;
            t2 = rRe * s->rSc + 0.0;
          }
          A_(sub, i, j, k) = -0.5 * rkdt * t1 * M(D->rdze, k - 1) * M(D->rdzc, k);
          A_(sup, i, j, k) = -0.5 * rkdt * t2 * M(D->rdze, k) * M(D->rdzc, k);
          A_(diag, i, j, k) =
              1.0 + 0.5 * rkdt * (t1 * M(D->rdze, k - 1) + t2 * M(D->rdze, k)) * M(D->rdzc, k);
        }
        if (les_var && i >= 1 && j >= 1) {
          for (int k = sz; k <= ez; ++k) {
            const double ra1 = H * (A_(r, i, j, k + 1) + A_(r, i, j, k));
            const double ra2 = H * (A_(r, i, j, k) + A_(r, i, j, k - 1));
            double t1, t2;
            if (var == 1) {
              t1 = -0.25 * (A_(kT, i, j, k) + A_(kT, i + 1 <= D->X ? i + 1 : i, j, k) +
                            A_(kT, i, j, k - 1) + A_(kT, i + 1 <= D->X ? i + 1 : i, j, k - 1)) *
                   ra1 / A_(r, i, j, k);
              t2 = -0.25 * (A_(kT, i, j, k) + A_(kT, i + 1 <= D->X ? i + 1 : i, j, k) +
                            A_(kT, i, j, k + 1) + A_(kT, i + 1 <= D->X ? i + 1 : i, j, k + 1)) *
                   ra2 / A_(r, i, j, k);
            } else if (var == 2) {
              t1 = -0.25 * (A_(kT, i, j, k) + A_(kT, i, j + 1 <= D->Y ? j + 1 : j, k) +
                            A_(kT, i, j, k - 1) + A_(kT, i, j + 1 <= D->Y ? j + 1 : j, k - 1)) *
                   ra1 / A_(r, i, j, k);
              t2 = -0.25 * (A_(kT, i, j, k) + A_(kT, i, j + 1 <= D->Y ? j + 1 : j, k) +
                            A_(kT, i, j, k + 1) + A_(kT, i, j + 1 <= D->Y ? j + 1 : j, k + 1)) *
                   ra2 / A_(r, i, j, k);
            } else if (var == 5) {
              t1 = -0.5 * (A_(kT, i, j, k) + A_(kT, i, j, k - 1)) * ra1 / A_(r, i, j, k);
              t2 = -0.5 * (A_(kT, i, j, k) + A_(kT, i, j, k + 1)) * ra2 / A_(r, i, j, k);
            } else {
              t1 = -0.5 * (A_(kT, i, j, k) + A_(kT, i, j, k - 1));
              t2 = -0.5 * (A_(kT, i, j, k) + A_(kT, i, j, k + 1));
            }
            A_(sub, i, j, k) = A_(sub, i, j, k) - 1 * 0.5 * rkdt * t1 * M(D->rdze, k - 1) * M(D->rdzc, k);
            A_(sup, i, j, k) = A_(sup, i, j, k) - 1 * 0.5 * rkdt * t2 * M(D->rdze, k) * M(D->rdzc, k);
            A_(diag, i, j, k) = A_(diag, i, j, k) + 1 * 0.5 * rkdt *
                                                        (t1 * M(D->rdze, k - 1) + t2 * M(D->rdze, k)) *
                                                        M(D->rdzc, k);
          }
        }
      } else {
        for (int k = sz; k <= ez; ++k) {
          const double t1 = (rRe + 0.0) * A_(r, i, j, k) / (H * (A_(r, i, j, k + 1) + A_(r, i, j, k)));
          const double t2 =
              (rRe + 0.0) * A_(r, i, j, k + 1) / (H * (A_(r, i, j, k + 1) + A_(r, i, j, k)));
          A_(sub, i, j, k) = -0.5 * rkdt * t1 * M(D->rdze, k) * M(D->rdzc, k);
          A_(sup, i, j, k) = -0.5 * rkdt * t2 * M(D->rdze, k) * M(D->rdzc, k + 1);
          A_(diag, i, j, k) =
              1.0 + 0.5 * rkdt * (t1 * M(D->rdzc, k) + t2 * M(D->rdzc, k + 1)) * M(D->rdze, k);
        }
        if (les) {
          for (int k = sz; k <= ez; ++k) {
            const double t1 =
                -A_(kT, i, j, k) * A_(r, i, j, k) / (H * (A_(r, i, j, k + 1) + A_(r, i, j, k)));
            const double t2 =
                -A_(kT, i, j, k + 1) * A_(r, i, j, k + 1) / (H * (A_(r, i, j, k + 1) + A_(r, i, j, k)));
            A_(sub, i, j, k) = A_(sub, i, j, k) - 1 * 1.0 * rkdt * t1 * M(D->rdze, k) * M(D->rdzc, k);
            A_(sup, i, j, k) =
                A_(sup, i, j, k) - 1 * 1.0 * rkdt * t2 * M(D->rdze, k) * M(D->rdzc, k + 1);
            A_(diag, i, j, k) = A_(diag, i, j, k) + 1 * 1.0 * rkdt *
                                                        (t1 * M(D->rdzc, k) + t2 * M(D->rdzc, k + 1)) *
                                                        M(D->rdze, k);
          }
        }
      }
    }
  /* right-hand side (:3185-3296) */
#pragma omp parallel for schedule(static)
  for (long j = 1; j <= D->Y; ++j)
    for (long i = 1; i <= D->X; ++i)
      for (int k = sz; k <= ez; ++k) {
        A_(rhs, i, j, k) = 1.0 * A_(u, i, j, k) + a3 * A_(q, i, j, k) * 1.0;
        if (var != 3) {
          const double ra1 = H * (A_(r, i, j, k + 1) + A_(r, i, j, k));
          const double ra2 = H * (A_(r, i, j, k) + A_(r, i, j, k - 1));
          double t1, t2;
          if (var == 1 || var == 2) {
            t1 = (rRe + 0.0) * ra1 / A_(r, i, j, k);
            t2 = (rRe + 0.0) * ra2 / A_(r, i, j, k);
          } else if (var == 5) {
            t1 = (rRe * s->rPr + 0.0) * ra1 / A_(r, i, j, k);
            t2 = (rRe * s->rPr + 0.0) * ra2 / A_(r, i, j, k);
          } else {
            t1 = rRe * s->rSc + 0.0;
            t2 = rRe * s->rSc + 0.0;
          }
          A_(rhs, i, j, k) =
              A_(rhs, i, j, k) +
              rkdt * 0.5 *
                  (t2 * (A_(u, i, j, k + 1) - A_(u, i, j, k)) * M(D->rdze, k) -
                   t1 * (A_(u, i, j, k) - A_(u, i, j, k - 1)) * M(D->rdze, k - 1)) *
                  M(D->rdzc, k);
          if (les_var) {
            if (var == 1) {
              const long ip = i + 1 <= D->X ? i + 1 : i;
              t1 = -0.25 * (A_(kT, i, j, k) + A_(kT, ip, j, k) + A_(kT, i, j, k - 1) + A_(kT, ip, j, k - 1)) *
                   ra1 / A_(r, i, j, k);
              t2 = -0.25 * (A_(kT, i, j, k) + A_(kT, ip, j, k) + A_(kT, i, j, k + 1) + A_(kT, ip, j, k + 1)) *
                   ra2 / A_(r, i, j, k);
            } else if (var == 2) {
              const long jp = j + 1 <= D->Y ? j + 1 : j;
              t1 = -0.25 * (A_(kT, i, j, k) + A_(kT, i, jp, k) + A_(kT, i, j, k - 1) + A_(kT, i, jp, k - 1)) *
                   ra1 / A_(r, i, j, k);
              t2 = -0.25 * (A_(kT, i, j, k) + A_(kT, i, jp, k) + A_(kT, i, j, k + 1) + A_(kT, i, jp, k + 1)) *
                   ra2 / A_(r, i, j, k);
            } else if (var == 5) {
              t1 = -0.5 * (A_(kT, i, j, k) + A_(kT, i, j, k - 1)) * ra1 / A_(r, i, j, k);
              t2 = -0.5 * (A_(kT, i, j, k) + A_(kT, i, j, k + 1)) * ra2 / A_(r, i, j, k);
            } else {
              t1 = -0.5 * (A_(kT, i, j, k) + A_(kT, i, j, k - 1));
              t2 = -0.5 * (A_(kT, i, j, k) + A_(kT, i, j, k + 1));
            }
            A_(rhs, i, j, k) =
                A_(rhs, i, j, k) +
                1 * rkdt * 0.5 *
                    (t2 * (A_(u, i, j, k + 1) - A_(u, i, j, k)) * M(D->rdze, k) -
                     t1 * (A_(u, i, j, k) - A_(u, i, j, k - 1)) * M(D->rdze, k - 1)) *
                    M(D->rdzc, k);
          }
        } else {
          const double t1 = (rRe + 0.0) * A_(r, i, j, k) / (H * (A_(r, i, j, k + 1) + A_(r, i, j, k)));
          const double t2 =
              (rRe + 0.0) * A_(r, i, j, k + 1) / (H * (A_(r, i, j, k + 1) + A_(r, i, j, k)));
          A_(rhs, i, j, k) =
              A_(rhs, i, j, k) +
              rkdt * 0.5 *
                  (t2 * (A_(u, i, j, k + 1) - A_(u, i, j, k)) * M(D->rdzc, k + 1) -
                   t1 * (A_(u, i, j, k) - A_(u, i, j, k - 1)) * M(D->rdzc, k)) *
                  M(D->rdze, k);
          if (les) {
            const double u1 = -A_(kT, i, j, k) * A_(r, i, j, k) / (H * (A_(r, i, j, k + 1) + A_(r, i, j, k)));
            const double u2 =
                -A_(kT, i, j, k + 1) * A_(r, i, j, k + 1) / (H * (A_(r, i, j, k + 1) + A_(r, i, j, k)));
            A_(rhs, i, j, k) =
                A_(rhs, i, j, k) +
                1 * rkdt * 1.0 *
                    (u2 * (A_(u, i, j, k + 1) - A_(u, i, j, k)) * M(D->rdzc, k + 1) -
                     u1 * (A_(u, i, j, k) - A_(u, i, j, k - 1)) * M(D->rdzc, k)) *
                    M(D->rdze, k);
          }
        }
      }
  ghost(s, sub, VT_CFLUC);
  ghost(s, diag, VT_CFLUC);
  ghost(s, sup, VT_CFLUC);
  ghost(s, rhs, VT_CFLUC);
  /* wall rows (:3297-3429) */
  const int tbmin = s->p.tb[2][0][var - 1], tbmax = s->p.tb[2][1][var - 1];
  const double vbmin = s->p.vb[2][0][var - 1], vbmax = s->p.vb[2][1][var - 1];
  for (long j = 1; j <= D->Y; ++j)
    for (long i = 1; i <= D->X; ++i) {
#define SET(k, a, b, c, d) \
  do {                     \
    A_(sub, i, j, k) = a;  \
    A_(diag, i, j, k) = b; \
    A_(sup, i, j, k) = c;  \
    A_(rhs, i, j, k) = d;  \
  } while (0)
      if (tbmin == 1) SET(sz - 1, 0.0, 1.0, 0.0, vbmin);
      else if (tbmin == 2) {
        if (var == 3) SET(sz - 1, 0.0, -1.0, 1.0, M(D->dzc, sz - 1) * vbmin);
        else if (var == 5 || var == 8) {
          SET(sz - 1, 0.0, -1.0, 1.0, M(D->dze, sz - 1) * vbmin);
          SET(sz, 0.0, -1.0, 1.0, M(D->dze, sz) * vbmin);
        } else SET(sz - 1, 0.0, -1.0, 1.0, M(D->dze, sz - 1) * vbmin);
      } else if (tbmin == 6) SET(sz - 1, 0.0, 1.0, 1.0, 2.0 * vbmin);
      if (tbmax == 1) SET(ez + 1, 0.0, 1.0, 0.0, vbmax);
      else if (tbmax == 2) {
        if (var == 3) SET(ez + 1, -1.0, 1.0, 0.0, M(D->dzc, ez + 1) * vbmax);
        else if (var == 5 || var == 8) {
          SET(ez + 1, -1.0, 1.0, 0.0, M(D->dze, ez + 1) * vbmax);
          SET(ez, -1.0, 1.0, 0.0, M(D->dze, ez) * vbmax);
        } else SET(ez + 1, -1.0, 1.0, 0.0, M(D->dze, ez + 1) * vbmax);
      } else if (tbmax == 6) SET(ez + 1, 1.0, 1.0, 0.0, 2.0 * vbmax);
      else if (tbmax == 7) {
        SET(ez + 1, 0.0, 1.0, 0.0, 0.0);
        SET(ez, 0.0, 1.0, 0.0, 0.0);
      }
#undef SET
    }
  /* Thomas per interior column over k = 1..nz+2 (:3431-3436) */
  const int n = D->nz + 2;
#pragma omp parallel for schedule(static)
  for (int j = 2; j <= D->ny + 1; ++j) {
    double* a = (double*)malloc(sizeof(double) * 4 * n);
    double *b = a + n, *cc = b + n, *gg = cc + n;
    for (int i = 2; i <= D->nx + 1; ++i) {
      for (int k = 1; k <= n; ++k) {
        a[k - 1] = A_(sub, i, j, k);
        b[k - 1] = A_(diag, i, j, k);
        cc[k - 1] = A_(sup, i, j, k);
        gg[k - 1] = A_(rhs, i, j, k);
      }
      thomas_ns(a, b, cc, gg, n);
      for (int k = 1; k <= n; ++k) A_(rhs, i, j, k) = gg[k - 1];
    }
    free(a);
  }
  ghost(s, rhs, var == 1 ? VT_U : var == 2 ? VT_V : var == 3 ? VT_W : var == 5 ? VT_RHO : VT_SCAL1);
  memcpy(u, rhs, sizeof(double) * G);
}

/* ---------------------------------------------------------------- Psource
 * NSsolver.F90:2167-2223 */
static void psource(orc_ns* s, double* SRC, double dt) {
  const orc_dom* D = &s->d;
  const double *U = s->f.u, *V = s->f.v, *W = s->f.w, *r = s->f.r;
  const double H = (double)(float)0.5;
  memset(SRC, 0, sizeof(double) * D->G);
  const double rdt = 1.0 / dt;
  #pragma omp parallel for schedule(static)
  for (int k = 2; k <= D->nz + 1; ++k)
    for (int j = 2; j <= D->ny + 1; ++j)
      for (int i = 2; i <= D->nx + 1; ++i)
        A_(SRC, i, j, k) =
            A_(SRC, i, j, k) +
            ((A_(r, i, j, k) * A_(U, i, j, k) - A_(r, i, j, k) * A_(U, i - 1, j, k)) * M(D->rdxc, i) +
             (A_(r, i, j, k) * A_(V, i, j, k) - A_(r, i, j, k) * A_(V, i, j - 1, k)) * M(D->rdyc, j) +
             (H * (A_(r, i, j, k + 1) + A_(r, i, j, k)) * A_(W, i, j, k) -
              H * (A_(r, i, j, k) + A_(r, i, j, k - 1)) * A_(W, i, j, k - 1)) *
                 M(D->rdzc, k)) *
                rdt;
  ghost(s, SRC, VT_PSOURCE);
}

/* ---------------------------------------------------------------- Pgrad
 * NSsolver.F90:2023-2085 */
static void pgrad(orc_ns* s, double dt) {
  const orc_dom* D = &s->d;
  const double *pn = s->f.p, *r = s->f.r;
  double *U = s->f.u, *V = s->f.v, *W = s->f.w;
  #pragma omp parallel for schedule(static)
  for (int k = 2; k <= D->nz + 1; ++k)
    for (int j = 2; j <= D->ny + 1; ++j)
      for (int i = 2; i <= D->nx + 1; ++i)
        A_(U, i, j, k) = A_(U, i, j, k) - (A_(pn, i + 1, j, k) / A_(r, i, j, k) -
                                           A_(pn, i, j, k) / A_(r, i, j, k)) *
                                              M(D->rdxe, i) * dt;
  ghost(s, U, VT_UTEMP);
  #pragma omp parallel for schedule(static)
  for (int k = 2; k <= D->nz + 1; ++k)
    for (int j = 2; j <= D->ny + 1; ++j)
      for (int i = 2; i <= D->nx + 1; ++i)
        A_(V, i, j, k) = A_(V, i, j, k) - (A_(pn, i, j + 1, k) / A_(r, i, j, k) -
                                           A_(pn, i, j, k) / A_(r, i, j, k)) *
                                              M(D->rdye, j) * dt;
  ghost(s, V, VT_VTEMP);
  #pragma omp parallel for schedule(static)
  for (int k = 2; k <= D->nz + 1 - s->p.ew; ++k)
    for (int j = 2; j <= D->ny + 1; ++j)
      for (int i = 2; i <= D->nx + 1; ++i)
        A_(W, i, j, k) = A_(W, i, j, k) - (A_(pn, i, j, k + 1) / A_(r, i, j, k + 1) -
                                           A_(pn, i, j, k) / A_(r, i, j, k)) *
                                              M(D->rdze, k) * dt;
  ghost(s, W, VT_WTEMP);
}

/* ---------------------------------------------------------------- rk_ss
 * NSsolver.F90:418-583 (RK3CN branch). */
int orc_ns_substep(orc_ns* s, double a1, double a2, double a3, double dt_rk, double dt, int* iters,
                   double* relmax) {
  const orc_dom* D = &s->d;
  anel_fields* f = &s->f;
  memset(f->psrc, 0, sizeof(double) * D->G);
  u1_rhs(s, s->Ftemp);
  var_advance(s, s->Ftemp, f->q_u, a1, a2, dt);
  u2_rhs(s, s->Ftemp);
  var_advance(s, s->Ftemp, f->q_v, a1, a2, dt);
  u3_rhs(s, s->Ftemp);
  var_advance(s, s->Ftemp, f->q_w, a1, a2, dt);
  scalar_rhs(s, s->Ftemp, 1);
  var_advance(s, s->Ftemp, f->q_rho, a1, a2, dt);
  scalar_rhs(s, s->Ftemp, 0);
  var_advance(s, s->Ftemp, f->q_s, a1, a2, dt);
  ghost(s, f->q_u, VT_UTEMP);
  ghost(s, f->q_v, VT_VTEMP);
  ghost(s, f->q_w, VT_WTEMP);
  ghost(s, f->q_rho, VT_RTEMP);
  ghost(s, f->q_s, VT_S1TEMP);
  cn_pl(s, f->q_u, f->u, a3, dt_rk, 1);
  cn_pl(s, f->q_v, f->v, a3, dt_rk, 2);
  cn_pl(s, f->q_w, f->w, a3, dt_rk, 3);
  memset(f->psrc, 0, sizeof(double) * D->G);
  psource(s, f->psrc, dt_rk);
  cn_pl(s, f->q_rho, f->rho, a3, dt_rk, 5);
  cn_pl(s, f->q_s, f->scal1, a3, dt_rk, 8);
  /* Ftemp = p ; mg_solver(Ftemp, r_tmp1, niters, resmax) ; p = Ftemp */
  memcpy(s->Ftemp, f->p, sizeof(double) * D->G);
  orc_mg_set_density(s->mg, f->r);
  orc_mg_solve(s->mg, s->Ftemp, f->psrc, iters, relmax);
  memcpy(f->p, s->Ftemp, sizeof(double) * D->G);
  pgrad(s, dt_rk);
  ghost(s, f->q_u, VT_UTEMP);
  ghost(s, f->q_v, VT_VTEMP);
  ghost(s, f->q_w, VT_WTEMP);
  ghost(s, f->u, VT_U);
  ghost(s, f->v, VT_V);
  ghost(s, f->w, VT_W);
  ghost(s, f->rho, VT_RHO);
  ghost(s, f->scal1, VT_SCAL1);
  return 0;
}

/* ---------------------------------------------------------------- calcdt
 * Routines.F90:186-258 and NSsolver.F90:72-73 */
static double calcdt(const orc_ns* s) {
  const orc_dom* D = &s->d;
  const double *u = s->f.u, *v = s->f.v, *w = s->f.w;
  double mx = 0.0;
  for (int k = 2; k <= D->nz + 1; ++k)
    for (int j = 2; j <= D->ny + 1; ++j)
      for (int i = 2; i <= D->nx + 1; ++i) {
        const double adv = M(D->rdxc, i) * fabs(0.5 * (A_(u, i, j, k) + A_(u, i - 1, j, k))) +
                           M(D->rdzc, k) * fabs(0.5 * (A_(w, i, j, k) + A_(w, i, j, k - 1))) +
                           M(D->rdyc, j) * fabs(0.5 * (A_(v, i, j, k) + A_(v, i, j - 1, k)));
        mx = mx > adv ? mx : adv;
      }
  double dt = s->p.cfl / mx;
  if (dt >= s->p.dtmax) dt = s->p.dtmax;
  return dt;
}

/* gravity ramp, Routines.F90:27-52 */
static void gravity(orc_ns* s) {
  const double t = s->time, t1 = s->p.gt1, t2 = s->p.gt2;
  if (t < t1) s->gnow = 0.0;
  else if (t > t1 && t < t2) s->gnow = s->g_orig * (t - t1) / (t2 - t1);
  else if (t >= t2) s->gnow = s->g_orig;
}

/* straincal's strain magnitude (straincal.F90:48-73) of (l1, l2, l3) into
 * modS, ghost 'cfluc' */
static void modS_of(orc_ns* s, const double* l1, const double* l2, const double* l3, double* modS) {
  const orc_dom* D = &s->d;
  memset(modS, 0, sizeof(double) * D->G);
  for (int k = 2; k <= D->nz + 1; ++k)
    for (int j = 2; j <= D->ny + 1; ++j)
      for (int i = 2; i <= D->nx + 1; ++i) {
        const double TS11 = (A_(l1, i + 1, j, k) - A_(l1, i, j, k)) * M(D->rdxc, i);
        const double TS22 = (A_(l2, i, j + 1, k) - A_(l2, i, j, k)) * M(D->rdyc, j);
        const double TS33 = (A_(l3, i, j, k + 1) - A_(l3, i, j, k)) * M(D->rdzc, k);
        double t1 = 0.25 * (A_(l1, i, j, k) + A_(l1, i + 1, j, k) + A_(l1, i, j + 1, k) + A_(l1, i + 1, j + 1, k));
        double t2 = 0.25 * (A_(l1, i, j, k) + A_(l1, i + 1, j, k) + A_(l1, i, j - 1, k) + A_(l1, i + 1, j - 1, k));
        double t3 = 0.25 * (A_(l2, i, j, k) + A_(l2, i, j + 1, k) + A_(l2, i + 1, j, k) + A_(l2, i + 1, j + 1, k));
        double t4 = 0.25 * (A_(l2, i, j, k) + A_(l2, i, j + 1, k) + A_(l2, i - 1, j, k) + A_(l2, i - 1, j + 1, k));
        const double TS12 = 0.5 * ((t1 - t2) * M(D->rdyc, j) + (t3 - t4) * M(D->rdxc, i));
        t1 = 0.25 * (A_(l1, i, j, k) + A_(l1, i + 1, j, k) + A_(l1, i, j, k + 1) + A_(l1, i + 1, j, k + 1));
        t2 = 0.25 * (A_(l1, i, j, k) + A_(l1, i + 1, j, k) + A_(l1, i, j, k - 1) + A_(l1, i + 1, j, k - 1));
        t3 = 0.25 * (A_(l3, i, j, k) + A_(l3, i, j, k + 1) + A_(l3, i + 1, j, k) + A_(l3, i + 1, j, k + 1));
        t4 = 0.25 * (A_(l3, i, j, k) + A_(l3, i, j, k + 1) + A_(l3, i - 1, j, k) + A_(l3, i - 1, j, k + 1));
        const double TS13 = 0.5 * ((t1 - t2) * M(D->rdzc, k) + (t3 - t4) * M(D->rdxc, i));
        t1 = 0.25 * (A_(l2, i, j, k) + A_(l2, i, j + 1, k) + A_(l2, i, j, k + 1) + A_(l2, i, j + 1, k + 1));
        t2 = 0.25 * (A_(l2, i, j, k) + A_(l2, i, j + 1, k) + A_(l2, i, j, k - 1) + A_(l2, i, j + 1, k - 1));
        t3 = 0.25 * (A_(l3, i, j, k) + A_(l3, i, j, k + 1) + A_(l3, i, j + 1, k) + A_(l3, i, j + 1, k + 1));
        t4 = 0.25 * (A_(l3, i, j, k) + A_(l3, i, j, k + 1) + A_(l3, i, j - 1, k) + A_(l3, i, j - 1, k + 1));
        const double TS23 = 0.5 * ((t1 - t2) * M(D->rdzc, k) + (t3 - t4) * M(D->rdyc, j));
        /* x**2.d0 is evaluated as x*x */
        A_(modS, i, j, k) = sqrt(2.0) * sqrt(TS11 * TS11 + TS22 * TS22 + TS33 * TS33 + 2.0 * (TS12 * TS12) +
                                             2.0 * (TS13 * TS13) + 2.0 * (TS23 * TS23));
      }
  ghost(s, modS, VT_CFLUC);
}

/* straincal modS of the current velocity */
static void straincal(orc_ns* s) { modS_of(s, s->f.u, s->f.v, s->f.w, s->modS); }

static void center_velocity(orc_ns* s, const double* in, double* out, int dir, int stretched,
                            int corrected);
static void avg_x1x2(orc_ns* s, double* var, double* outm, int vt);

/* ------------------------------------------------------ dynamic models
 * DSM (les/DSM.F90:1-258), DSMrho and DSMscal1 (les/DSMrho.F90,
 * DSMscal1.F90) with C_avg_dir = 12: the model coefficients are x-y plane
 * averages (LagAvg is not reached).  Test filter: filter(.., 2, xfil,
 * yfil, zfil, ..) (les/filter.F90:1-149); smoothing of the coefficient:
 * filterHF(.., 2, 1, 1, 1, ..) (:152-288).  Whole-array Fortran
 * assignments are whole-array loops here (ghost cells included). */
static long dyn_G(const orc_ns* s) { return s->d.G; }

/* filter(var, out, 2, xfil, yfil, zfil, vt): per direction a pass of
 * weights (1/4, 1/2, 1/4) over the interior, written with the source's
 * zero weights and its boundary formulas (the upper one sums from the
 * ghost inwards), then ghost(out, vt). */
static void filter2(orc_ns* s, const double* var, double* out, int vt) {
  const orc_dom* D = &s->d;
  static const double wa[5] = {0.0, 1.0 / 4.0, 1.0 / 2.0, 1.0 / 4.0, 0.0};
  static const double wab[5] = {1.0 / 4.0, 1.0 / 2.0, 1.0 / 4.0, 0.0, 0.0};
  memcpy(out, var, sizeof(double) * D->G);
  const int n[3] = {D->nx, D->ny, D->nz};
  double pen[4096];
  for (int d = 0; d < 3; ++d) {
    if (s->p.filt[d]) {
      const long st = d == 0 ? 1 : (d == 1 ? D->X : D->X * D->Y);
      const int sa = 2, ea = n[d] + 1;
      for (int k = 2; k <= D->nz + 1; ++k)
        for (int j = 2; j <= D->ny + 1; ++j)
          for (int i = 2; i <= D->nx + 1; ++i) {
            const int q = d == 0 ? i : (d == 1 ? j : k);
            if (q != 2) continue; /* one pencil per (other two indices) */
            const long b = IX(i, j, k) - (long)q * st;
            for (int t = sa - 1; t <= ea + 1; ++t) pen[t] = out[b + (long)t * st];
            for (int t = sa + 1; t <= ea - 1; ++t)
              out[b + (long)t * st] = wa[0] * pen[t - 2] + wa[1] * pen[t - 1] + wa[2] * pen[t] +
                                      wa[3] * pen[t + 1] + wa[4] * pen[t + 2];
            out[b + (long)sa * st] = wab[0] * pen[sa - 1] + wab[1] * pen[sa] + wab[2] * pen[sa + 1] +
                                     wab[3] * pen[sa + 2] + wab[4] * pen[sa + 3];
            out[b + (long)ea * st] = wab[0] * pen[ea + 1] + wab[1] * pen[ea] + wab[2] * pen[ea - 1] +
                                     wab[3] * pen[ea - 2] + wab[4] * pen[ea - 3];
          }
    }
    ghost(s, out, vt);
  }
}

/* filterHF(var, out, 2, 1, 1, 1, vt, ..): in each direction a point that
 * is a strict local extremum of its pencil takes the 3-point average when
 * that average is still an extremum of the same kind. */
static void filterHF2(orc_ns* s, const double* var, double* out, int vt) {
  const orc_dom* D = &s->d;
  static const double wa[3] = {1.0 / 4.0, 1.0 / 2.0, 1.0 / 4.0};
  memcpy(out, var, sizeof(double) * D->G);
  const int n[3] = {D->nx, D->ny, D->nz};
  double pen[4096];
  for (int d = 0; d < 3; ++d) {
    const long st = d == 0 ? 1 : (d == 1 ? D->X : D->X * D->Y);
    const int sa = 2, ea = n[d] + 1;
    for (int k = 2; k <= D->nz + 1; ++k)
      for (int j = 2; j <= D->ny + 1; ++j)
        for (int i = 2; i <= D->nx + 1; ++i) {
          const int q = d == 0 ? i : (d == 1 ? j : k);
          if (q != 2) continue;
          const long b = IX(i, j, k) - (long)q * st;
          for (int t = sa - 1; t <= ea + 1; ++t) pen[t] = out[b + (long)t * st];
          for (int t = sa; t <= ea; ++t) {
            const double p0 = pen[t], pm = pen[t - 1], pp = pen[t + 1];
            if (p0 < pp && p0 < pm) {
              const double x = wa[0] * pm + wa[1] * p0 + wa[2] * pp;
              if (x < pp && x < pm) out[b + (long)t * st] = x;
            } else if (p0 > pp && p0 > pm) {
              const double x = wa[0] * pm + wa[1] * p0 + wa[2] * pp;
              if (x > pp && x > pm) out[b + (long)t * st] = x;
            }
          }
        }
    ghost(s, out, vt);
  }
}

/* DSM's lestmp1 for component ij (DSM.F90:38-86): the diagonal strain, and
 * for ij = 4..6 half the difference of the two cross derivatives (the
 * source subtracts where straincal adds). */
static double dsm_component(const orc_dom* D, const double* l1, const double* l2, const double* l3, int ij,
                            int i, int j, int k) {
  double t1, t2, t3, t4;
  switch (ij) {
    case 1: return (A_(l1, i + 1, j, k) - A_(l1, i, j, k)) * M(D->rdxc, i);
    case 2: return (A_(l2, i, j + 1, k) - A_(l2, i, j, k)) * M(D->rdyc, j);
    case 3: return (A_(l3, i, j, k + 1) - A_(l3, i, j, k)) * M(D->rdzc, k);
    case 4:
      t1 = 0.25 * (A_(l1, i, j, k) + A_(l1, i + 1, j, k) + A_(l1, i, j + 1, k) + A_(l1, i + 1, j + 1, k));
      t2 = 0.25 * (A_(l1, i, j, k) + A_(l1, i + 1, j, k) + A_(l1, i, j - 1, k) + A_(l1, i + 1, j - 1, k));
      t3 = 0.25 * (A_(l2, i, j, k) + A_(l2, i, j + 1, k) + A_(l2, i + 1, j, k) + A_(l2, i + 1, j + 1, k));
      t4 = 0.25 * (A_(l2, i, j, k) + A_(l2, i, j + 1, k) + A_(l2, i - 1, j, k) + A_(l2, i - 1, j + 1, k));
      return 0.5 * ((t1 - t2) * M(D->rdyc, j) - (t3 - t4) * M(D->rdxc, i));
    case 5:
      t1 = 0.25 * (A_(l1, i, j, k) + A_(l1, i + 1, j, k) + A_(l1, i, j, k + 1) + A_(l1, i + 1, j, k + 1));
      t2 = 0.25 * (A_(l1, i, j, k) + A_(l1, i + 1, j, k) + A_(l1, i, j, k - 1) + A_(l1, i + 1, j, k - 1));
      t3 = 0.25 * (A_(l3, i, j, k) + A_(l3, i, j, k + 1) + A_(l3, i + 1, j, k) + A_(l3, i + 1, j, k + 1));
      t4 = 0.25 * (A_(l3, i, j, k) + A_(l3, i, j, k + 1) + A_(l3, i - 1, j, k) + A_(l3, i - 1, j, k + 1));
      return 0.5 * ((t1 - t2) * M(D->rdzc, k) - (t3 - t4) * M(D->rdxc, i));
    default:
      t1 = 0.25 * (A_(l2, i, j, k) + A_(l2, i, j + 1, k) + A_(l2, i, j, k + 1) + A_(l2, i, j + 1, k + 1));
      t2 = 0.25 * (A_(l2, i, j, k) + A_(l2, i, j + 1, k) + A_(l2, i, j, k - 1) + A_(l2, i, j + 1, k - 1));
      t3 = 0.25 * (A_(l3, i, j, k) + A_(l3, i, j, k + 1) + A_(l3, i, j + 1, k) + A_(l3, i, j + 1, k + 1));
      t4 = 0.25 * (A_(l3, i, j, k) + A_(l3, i, j, k + 1) + A_(l3, i, j - 1, k) + A_(l3, i, j - 1, k + 1));
      return 0.5 * ((t1 - t2) * M(D->rdzc, k) - (t3 - t4) * M(D->rdyc, j));
  }
}

typedef struct {
  double *modS, *fmodS, *c[3], *fc[3], *l1, *l2, *l3, *l4, *P, *a, *b;
} dyn_work;

static double* dyn_alloc(const orc_ns* s) { return (double*)calloc(dyn_G(s), sizeof(double)); }

/* the fields every dynamic model starts from: straincal's modS and fmodS
 * (the strain magnitude of the filtered velocity, get_fmodS,
 * straincal.F90:166-229), the centred velocities and their filtered
 * forms (center_velocity, then filter(.., 'cfluc')) */
static void dyn_prepare(orc_ns* s, dyn_work* w) {
  anel_fields* f = &s->f;
  w->modS = dyn_alloc(s);
  w->fmodS = dyn_alloc(s);
  w->l1 = dyn_alloc(s);
  w->l2 = dyn_alloc(s);
  w->l3 = dyn_alloc(s);
  w->l4 = dyn_alloc(s);
  w->P = dyn_alloc(s);
  w->a = dyn_alloc(s);
  w->b = dyn_alloc(s);
  modS_of(s, f->u, f->v, f->w, w->modS);
  filter2(s, f->u, w->l1, VT_U);
  filter2(s, f->v, w->l2, VT_V);
  filter2(s, f->w, w->l3, VT_W);
  modS_of(s, w->l1, w->l2, w->l3, w->fmodS);
  const double* vel[3] = {f->u, f->v, f->w};
  for (int d = 0; d < 3; ++d) {
    w->c[d] = dyn_alloc(s);
    w->fc[d] = dyn_alloc(s);
    center_velocity(s, vel[d], w->c[d], d + 1, s->p.stretched[d], s->p.interp == ANEL_DIAG_CORRECTED);
    filter2(s, w->c[d], w->fc[d], VT_CFLUC);
  }
}

static void dyn_free(dyn_work* w) {
  double* p[] = {w->modS, w->fmodS, w->l1, w->l2, w->l3, w->l4, w->P, w->a, w->b,
                 w->c[0], w->c[1], w->c[2], w->fc[0], w->fc[1], w->fc[2]};
  for (unsigned q = 0; q < sizeof(p) / sizeof(p[0]); ++q) free(p[q]);
}

/* the plane averaging and ratio common to the three models (DSM.F90:
 * 196-256, DSMrho.F90:166-240): num and den are averaged over x-y planes,
 * the interior takes the plane values (num clipped at 0), then
 * out = 0.5 num / den (1e-20 where den == 0), smoothed by filterHF */
static void dyn_ratio(orc_ns* s, double* num, double* den, double* out, dyn_work* w) {
  const orc_dom* D = &s->d;
  const long Z = D->Z;
  double* pn = (double*)calloc(Z, sizeof(double));
  double* pd = (double*)calloc(Z, sizeof(double));
  ghost(s, num, VT_CFLUC);
  ghost(s, den, VT_CFLUC);
  avg_x1x2(s, num, pn, VT_CFLUC);
  avg_x1x2(s, den, pd, VT_CFLUC);
  for (int k = 2; k <= D->nz + 1; ++k)
    for (int j = 2; j <= D->ny + 1; ++j)
      for (int i = 2; i <= D->nx + 1; ++i) {
        A_(num, i, j, k) = pn[k - 1];
        A_(den, i, j, k) = pd[k - 1];
        if (A_(num, i, j, k) < 0.0) A_(num, i, j, k) = 0.0;
      }
  ghost(s, num, VT_CFLUC);
  ghost(s, den, VT_CFLUC);
  for (int k = 2; k <= D->nz + 1; ++k)
    for (int j = 2; j <= D->ny + 1; ++j)
      for (int i = 2; i <= D->nx + 1; ++i) {
        if (A_(den, i, j, k) == 0.0) A_(out, i, j, k) = 1.0e-20;
        else A_(out, i, j, k) = 0.5 * A_(num, i, j, k) / A_(den, i, j, k);
      }
  ghost(s, out, VT_CFLUC);
  filterHF2(s, out, w->P, VT_CFLUC);
  memcpy(out, w->P, sizeof(double) * D->G);
  ghost(s, out, VT_CFLUC);
  free(pn);
  free(pd);
}

/* DSM (DSM.F90:1-258) into Csgs */
static void dsm(orc_ns* s, double* Csgs) {
  const orc_dom* D = &s->d;
  const long G = D->G;
  const anel_fields* f = &s->f;
  dyn_work w;
  dyn_prepare(s, &w);
  const double rt = s->p.test_ratio;
  double *l1 = w.l1, *l2 = w.l2, *l3 = w.l3, *l4 = w.l4;
  memset(l4, 0, sizeof(double) * G);
  memset(Csgs, 0, sizeof(double) * G);
  static const int pa[7] = {0, 0, 1, 2, 0, 0, 1}, pb[7] = {0, 0, 1, 2, 1, 2, 2};
  for (int ij = 1; ij <= 6; ++ij) {
    for (int k = 2; k <= D->nz + 1; ++k)
      for (int j = 2; j <= D->ny + 1; ++j)
        for (int i = 2; i <= D->nx + 1; ++i) A_(l1, i, j, k) = dsm_component(D, f->u, f->v, f->w, ij, i, j, k);
    ghost(s, l1, VT_CFLUC);
    for (int k = 2; k <= D->nz + 1; ++k)
      for (int j = 2; j <= D->ny + 1; ++j)
        for (int i = 2; i <= D->nx + 1; ++i) {
          const double dg = A_(s->delg, i, j, k);
          A_(l2, i, j, k) = (dg * dg) * A_(w.modS, i, j, k) * A_(l1, i, j, k);
        }
    ghost(s, l2, VT_CFLUC);
    filter2(s, l2, l3, VT_CFLUC);
    filter2(s, l1, l2, VT_CFLUC);
    memcpy(l1, w.fmodS, sizeof(double) * G);
    for (int k = 2; k <= D->nz + 1; ++k)
      for (int j = 2; j <= D->ny + 1; ++j)
        for (int i = 2; i <= D->nx + 1; ++i) {
          const double rd = rt * A_(s->delg, i, j, k);
          A_(l2, i, j, k) = (rd * rd) * A_(l1, i, j, k) * A_(l2, i, j, k);
        }
    ghost(s, l2, VT_CFLUC);
    for (long c = 0; c < G; ++c) l3[c] = l3[c] - l2[c];
    ghost(s, l3, VT_CFLUC);
    const double *ca = w.c[pa[ij]], *cb = w.c[pb[ij]];
    for (long c = 0; c < G; ++c) w.a[c] = ca[c] * cb[c];
    filter2(s, w.a, l2, VT_CFLUC);
    const double *fa = w.fc[pa[ij]], *fb = w.fc[pb[ij]];
    if (ij <= 3) {
      for (long c = 0; c < G; ++c) l4[c] = l4[c] + l3[c] * l2[c];
      for (long c = 0; c < G; ++c) l4[c] = l4[c] - l3[c] * fa[c] * fb[c];
      for (long c = 0; c < G; ++c) Csgs[c] = Csgs[c] + l3[c] * l3[c];
    } else {
      for (long c = 0; c < G; ++c) l4[c] = l4[c] + 2.0 * l3[c] * l2[c];
      for (long c = 0; c < G; ++c) l4[c] = l4[c] - 2.0 * l3[c] * fa[c] * fb[c];
      for (long c = 0; c < G; ++c) Csgs[c] = Csgs[c] + 2.0 * l3[c] * l3[c];
    }
  }
  /* Csgs = 0.5 <LM> / <MM> */
  memcpy(w.b, Csgs, sizeof(double) * G);
  dyn_ratio(s, l4, w.b, Csgs, &w);
  dyn_free(&w);
}

/* DSMrho / DSMscal1 (DSMrho.F90:1-240) of the scalar c into C */
static void dsm_scalar(orc_ns* s, const double* c, double* C) {
  const orc_dom* D = &s->d;
  const long G = D->G;
  const anel_fields* f = &s->f;
  dyn_work w;
  dyn_prepare(s, &w);
  const double rt = s->p.test_ratio;
  double *l1 = w.l1, *l2 = w.l2, *l3 = w.l3, *l4 = w.l4;
  memset(l4, 0, sizeof(double) * G);
  memset(C, 0, sizeof(double) * G);
  const double* vel[3] = {f->u, f->v, f->w};
  for (int ij = 1; ij <= 3; ++ij) {
    const long st = ij == 1 ? 1 : (ij == 2 ? D->X : D->X * D->Y);
    for (int pass = 0; pass < 2; ++pass) {
      for (int k = 2; k <= D->nz + 1; ++k)
        for (int j = 2; j <= D->ny + 1; ++j)
          for (int i = 2; i <= D->nx + 1; ++i) {
            const long o = IX(i, j, k);
            const double t1 = 0.5 * (c[o] + c[o - st]);
            const double t2 = 0.5 * (c[o] + c[o + st]);
            const double rd = ij == 1 ? M(D->rdxc, i) : (ij == 2 ? M(D->rdyc, j) : M(D->rdzc, k));
            const double dg = A_(s->delg, i, j, k);
            l1[o] = pass == 0 ? (dg * dg) * A_(w.modS, i, j, k) * (t2 - t1) * rd : (t2 - t1) * rd;
          }
      ghost(s, l1, VT_CFLUC);
      filter2(s, l1, pass == 0 ? l2 : l3, VT_CFLUC);
    }
    memcpy(l1, w.fmodS, sizeof(double) * G);
    for (int k = 2; k <= D->nz + 1; ++k)
      for (int j = 2; j <= D->ny + 1; ++j)
        for (int i = 2; i <= D->nx + 1; ++i) {
          const double rd = rt * A_(s->delg, i, j, k);
          A_(l2, i, j, k) = A_(l2, i, j, k) - (rd * rd) * A_(l1, i, j, k) * A_(l3, i, j, k);
        }
    ghost(s, l2, VT_CFLUC);
    for (int k = 2; k <= D->nz + 1; ++k)
      for (int j = 2; j <= D->ny + 1; ++j)
        for (int i = 2; i <= D->nx + 1; ++i) {
          const long o = IX(i, j, k);
          l1[o] = c[o] * 0.5 * (vel[ij - 1][o - st] + vel[ij - 1][o]);
        }
    ghost(s, l1, VT_CFLUC);
    filter2(s, l1, l3, VT_CFLUC);
    filter2(s, c, w.a, VT_CFLUC);
    for (long q = 0; q < G; ++q) l3[q] = l3[q] - w.a[q] * w.fc[ij - 1][q];
    ghost(s, l3, VT_CFLUC);
    for (long q = 0; q < G; ++q) l4[q] = l4[q] + l2[q] * l2[q];
    for (long q = 0; q < G; ++q) C[q] = C[q] + l2[q] * l3[q];
  }
  memcpy(w.b, C, sizeof(double) * G);
  dyn_ratio(s, w.b, l4, C, &w);
  dyn_free(&w);
}

/* grid-only LES quantities: delg (straincal.F90:126-134) and the model
 * coefficients Csgs/CTsgs/CSsgs (SSM.F90:27,60,97) */
static void les_coeffs(orc_ns* s) {
  const orc_dom* D = &s->d;
  for (int k = 2; k <= D->nz + 1; ++k)
    for (int j = 2; j <= D->ny + 1; ++j)
      for (int i = 2; i <= D->nx + 1; ++i) {
        double dg;
        if (s->p.les_delta == ANEL_DELTA_3ROOT)
          dg = pow(M(D->dxc, i) * M(D->dyc, j) * M(D->dzc, k), 1.0 / 3.0);
        else
          dg = pow(M(D->dxc, i) * M(D->dxc, i) + M(D->dyc, j) * M(D->dyc, j) + M(D->dzc, k) * M(D->dzc, k),
                   1.0 / 2.0);
        A_(s->delg, i, j, k) = dg;
        const double c = s->p.ssm_const;
        double damp_u, damp_t;
        if (s->p.les_damp == ANEL_DAMP_LITERAL) {
          const double k41 = (double)(float)0.41;
          const double zo_u = 0.3, zo_t = (double)(float)0.3; /* 0.3d0 in SSM, 0.3 in SSMrho */
          const double a = k41 * (M(D->zc, k) + zo_u);
          damp_u = (a * a) / ((a * a) + c * (dg * dg));
          const double b = k41 * (M(D->zc, k) + zo_t);
          damp_t = (b * b) / ((b * b) + c * (dg * dg));
        } else {
          damp_u = 1.0;
          damp_t = 1.0;
        }
        if (s->p.vmodel != ANEL_MODEL_DSM) A_(s->Csgs, i, j, k) = c * damp_u;
        A_(s->work[0], i, j, k) = damp_t;
        A_(s->work[1], i, j, k) = damp_u;
      }
  ghost(s, s->delg, VT_CFLUC);
  /* the driver's order (NSsolver.F90:83-130): the velocity model, then
   * SSMrho / SSMscal1 from its Csgs, or their dynamic forms */
  if (s->p.vmodel == ANEL_MODEL_DSM) dsm(s, s->Csgs);
  ghost(s, s->Csgs, VT_CFLUC);
  for (int q = 0; q < 2; ++q) {
    double* C = q == 0 ? s->CTsgs : s->CSsgs;
    const int model = q == 0 ? s->p.rmodel : s->p.smodel;
    if (model == ANEL_MODEL_DSM) {
      dsm_scalar(s, q == 0 ? s->f.rho : s->f.scal1, C);
    } else {
      for (int k = 2; k <= D->nz + 1; ++k)
        for (int j = 2; j <= D->ny + 1; ++j)
          for (int i = 2; i <= D->nx + 1; ++i)
            A_(C, i, j, k) = A_(s->Csgs, i, j, k) / s->p.pr_sgs * A_(s->work[q], i, j, k);
    }
    ghost(s, C, VT_CFLUC);
  }
}

/* SGSdiff (straincal.F90:339-414): nuT, kappaT, nappaT */
static void sgsdiff(orc_ns* s) {
  const orc_dom* D = &s->d;
  straincal(s);
  double* outs[3] = {s->f.nuT, s->f.kappaT, s->f.nappaT};
  const double* C[3] = {s->Csgs, s->CTsgs, s->CSsgs};
  for (int q = 0; q < 3; ++q) {
    double* o = outs[q];
    memset(o, 0, sizeof(double) * D->G);
    for (int k = 2; k <= D->nz + 1; ++k)
      for (int j = 2; j <= D->ny + 1; ++j)
        for (int i = 2; i <= D->nx + 1; ++i)
          A_(o, i, j, k) = -(A_(C[q], i, j, k) + 0.0) * (A_(s->delg, i, j, k) * A_(s->delg, i, j, k)) *
                               A_(s->modS, i, j, k) +
                           0.0;
    ghost(s, o, VT_CFLUC);
  }
}

/* One NSsolver time step (NSsolver.F90:63-283 minus output/statistics). */
/* clipVS (Routines.F90:301-380): interior values below vmin become vmin,
 * then values above vmax become vmax (the clipped-point counts it prints
 * are not kept). */
static void clip_vs(const orc_ns* s, double* var, double vmin, double vmax) {
  const orc_dom* D = &s->d;
  for (long k = 2; k <= D->nz + 1; ++k)
    for (long j = 2; j <= D->ny + 1; ++j)
      for (long i = 2; i <= D->nx + 1; ++i) {
        double* v = &var[IX(i, j, k)];
        if (*v < vmin) *v = vmin;
        if (*v > vmax) *v = vmax;
      }
}

int orc_ns_step(orc_ns* s, anel_step_report* rep) {
  const orc_dom* D = &s->d;
  anel_fields* f = &s->f;
  const long G = D->G;
  memset(f->q_u, 0, sizeof(double) * G);
  memset(f->q_v, 0, sizeof(double) * G);
  memset(f->q_w, 0, sizeof(double) * G);
  memset(f->psrc, 0, sizeof(double) * G);
  memset(f->q_rho, 0, sizeof(double) * G);
  memset(f->q_s, 0, sizeof(double) * G);
  const double delt = calcdt(s);
  gravity(s);
  const int les = s->p.vmodel != ANEL_MODEL_DNS;
  if (les && s->nstep >= s->p.les_start && s->nstep % s->p.les_freq == 0) les_coeffs(s);
  /* every 50 steps the scalar LES models smooth rho and scal1 with
   * filterHF(.., 2, 1, 1, 1, 'rho' / 'scal1', ..) (NSsolver.F90:144-164;
   * its EDIFF and tol arguments are unused, filter.F90:209,237,266): a
   * whole-array copy back, then the field's ghost pass */
  if (s->time > 0.0 && s->nstep % 50 == 0) {
    if (s->p.rmodel != ANEL_MODEL_DNS) {
      filterHF2(s, f->rho, s->work[3], VT_RHO);
      memcpy(f->rho, s->work[3], sizeof(double) * G);
      ghost(s, f->rho, VT_RHO);
    }
    if (s->p.smodel != ANEL_MODEL_DNS) {
      filterHF2(s, f->scal1, s->work[3], VT_SCAL1);
      memcpy(f->scal1, s->work[3], sizeof(double) * G);
      ghost(s, f->scal1, VT_SCAL1);
    }
  }
  static const double A1[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
  static const double A3[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
  const double DTR[3] = {1.0 / 3.0 * delt, 5.0 / 12.0 * delt, 1.0 / 4.0 * delt};
  int it[3];
  double rm[3];
  for (int q = 0; q < 3; ++q) {
    if (les && s->nstep > s->p.les_start) sgsdiff(s);
    orc_ns_substep(s, A1[q], 1.0, A3[q], DTR[q], delt, &it[q], &rm[q]);
    if (s->p.clip) { /* NSsolver.F90:206-211 (and :235-240, :264-269) */
      clip_vs(s, f->rho, s->p.rho_min, s->p.rho_max);
      ghost(s, f->rho, VT_RHO);
      clip_vs(s, f->scal1, s->p.scal1_min, s->p.scal1_max);
      ghost(s, f->scal1, VT_SCAL1);
    }
  }
  s->told = s->time; /* told = time; time = time + delt (NSsolver.F90:272-274) */
  s->time = s->time + delt;
  if (rep) {
    rep->nstep = s->nstep;
    rep->dt = delt;
    rep->time = s->time;
    for (int q = 0; q < 3; ++q) {
      rep->mg_iter[q] = it[q];
      rep->mg_relmax[q] = rm[q];
    }
  }
  s->nstep += 1;
  return 0;
}

/* Projection of the initial field (not a reference routine: the
 * shear-layer benchmark starts from a divergence-free field): velocity
 * ghosts, Psource with dt = 1, one MG solve from p, Pgrad with dt = 1,
 * velocity ghosts. */
int orc_ns_project(orc_ns* s, int* iters, double* relmax) {
  const orc_dom* D = &s->d;
  anel_fields* f = &s->f;
  /* velocity ghosts first, so the wall flux of Psource vanishes */
  ghost(s, f->u, VT_U);
  ghost(s, f->v, VT_V);
  ghost(s, f->w, VT_W);
  memset(f->psrc, 0, sizeof(double) * D->G);
  psource(s, f->psrc, 1.0);
  memcpy(s->Ftemp, f->p, sizeof(double) * D->G);
  orc_mg_set_density(s->mg, f->r);
  orc_mg_solve(s->mg, s->Ftemp, f->psrc, iters, relmax);
  memcpy(f->p, s->Ftemp, sizeof(double) * D->G);
  pgrad(s, 1.0);
  ghost(s, f->u, VT_U);
  ghost(s, f->v, VT_V);
  ghost(s, f->w, VT_W);
  return 0;
}

/* ghost() of one field by type name index (tests) */
void orc_ns_ghost(orc_ns* s, double* var, int vt) { ghost(s, var, vt); }

/* one Crank-Nicolson solve on caller arrays (tests) */
void orc_ns_cn(orc_ns* s, const double* q, double* u, double a3, double rkdt, int var) {
  cn_pl(s, q, u, a3, rkdt, var);
}

/* the LES update on the bound fields (tests) */
void orc_ns_les_update(orc_ns* s) {
  les_coeffs(s);
  sgsdiff(s);
}

/* one explicit right-hand side on the bound fields (tests) */
void orc_ns_rhs(orc_ns* s, int which, double* out) {
  gravity(s);
  switch (which) {
    case 0: u1_rhs(s, out); break;
    case 1: u2_rhs(s, out); break;
    case 2: u3_rhs(s, out); break;
    case 3: scalar_rhs(s, out, 1); break;
    default: scalar_rhs(s, out, 0); break;
  }
}

/* divergence (Routines.F90:54-183): out[0] avg, out[1] max |div| */
void orc_ns_divergence(orc_ns* s, double* out) {
  const orc_dom* D = &s->d;
  const double *u = s->f.u, *v = s->f.v, *w = s->f.w;
  double sum = 0.0, vol = 0.0, mx = 0.0;
  for (int k = 2; k <= D->nz + 1; ++k)
    for (int j = 2; j <= D->ny + 1; ++j)
      for (int i = 2; i <= D->nx + 1; ++i) {
        const double d = (A_(u, i, j, k) - A_(u, i - 1, j, k)) * M(D->rdxc, i) +
                         (A_(v, i, j, k) - A_(v, i, j - 1, k)) * M(D->rdyc, j) +
                         (A_(w, i, j, k) - A_(w, i, j, k - 1)) * M(D->rdzc, k);
        if (fabs(d) > mx) mx = fabs(d);
        sum = sum + fabs(d) / (M(D->rdxc, i) * M(D->rdyc, j) * M(D->rdzc, k));
        vol = vol + 1.0 / (M(D->rdxc, i) * M(D->rdyc, j) * M(D->rdzc, k));
      }
  out[0] = sum / vol;
  out[1] = mx;
}

/* ---------------------------------------------------- plane statistics
 * The driver's per-step dk/dt block (NSsolver.F90:288-395): cell-centred
 * velocities (center_velocity, StatTools.F90:87-289), x-y plane averages
 * (avgX1X2, Average.F90:279-368, summed in its j-outer, i-inner order),
 * the time derivatives of the mean profiles and of the second moments of
 * the fluctuations. */

/* divdiffs(x, y, a, 4) (StatTools.F90:563-609): divided differences of y
 * over the abscissae x. */
static void divdiffs4(const double* x, const double* y, double* a) {
  double Dm[5][5];
  for (int k = 0; k <= 4; ++k) Dm[k][0] = y[k];
  for (int j = 1; j <= 4; ++j)
    for (int k = j; k <= 4; ++k) Dm[k][j] = (Dm[k][j - 1] - Dm[k - 1][j - 1]) / (x[k] - x[k - j]);
  for (int k = 0; k <= 4; ++k) a[k] = Dm[k][k];
}

/* interpoly(dep, ind, loc, 4) (StatTools.F90:611-653).  As written
 * (corrected = 0) it passes the values as the abscissae of divdiffs and
 * steps the Newton form by (loc - dep(k)): the inverse interpolant,
 * evaluated at a coordinate.  corrected = 1 interpolates dep over ind. */
static double interpoly4(const double* dep, const double* ind, double loc, int corrected) {
  const double* x = corrected ? ind : dep;
  const double* y = corrected ? dep : ind;
  double a[5];
  divdiffs4(x, y, a);
  double sum1 = a[4];
  for (int k = 3; k >= 0; --k) sum1 = sum1 * (loc - x[k]) + a[k];
  return sum1;
}

/* center_velocity(Uin, Ucen, dir) (StatTools.F90:87-289): Ucen = 0, the
 * interior from the two faces (uniform axis) or the 5-point interpolation
 * (stretched axis; windows q-2..q+2, sx-1..sx+3 at sx, ex-3..ex+1 at ex),
 * then ghost(Ucen, 'u' / 'v' / 'w'). */
static void center_velocity(orc_ns* s, const double* in, double* out, int dir, int stretched,
                            int corrected) {
  const orc_dom* D = &s->d;
  memset(out, 0, sizeof(double) * D->G);
  const double* e = dir == 1 ? D->xe : (dir == 2 ? D->ye : D->ze);
  const double* c = dir == 1 ? D->xc : (dir == 2 ? D->yc : D->zc);
  const int n = dir == 1 ? D->nx : (dir == 2 ? D->ny : D->nz);
  const long st = dir == 1 ? 1 : (dir == 2 ? D->X : D->X * D->Y);
  for (int k = 2; k <= D->nz + 1; ++k)
    for (int j = 2; j <= D->ny + 1; ++j)
      for (int i = 2; i <= D->nx + 1; ++i) {
        const long o = IX(i, j, k);
        const int q = dir == 1 ? i : (dir == 2 ? j : k);
        if (!stretched) {
          out[o] = R12 * (in[o] + in[o - st]);
        } else {
          const int lo = q == 2 ? 1 : (q == n + 1 ? n - 2 : q - 2);
          double dep[5], ind[5];
          for (int m = 0; m < 5; ++m) {
            dep[m] = in[o + (long)(lo + m - q) * st];
            ind[m] = M(e, lo + m);
          }
          out[o] = interpoly4(dep, ind, M(c, q), corrected);
        }
      }
  ghost(s, out, dir == 1 ? VT_U : (dir == 2 ? VT_V : VT_W));
}

/* avgX1X2(Var, outm, vtype) for the cell-centred types (dxc, dyc
 * weights): ghost(Var, vt), then outm(k) = sum Var*dxc*dyc / Area for
 * k = sz-1..ez+1. */
static void avg_x1x2(orc_ns* s, double* var, double* outm, int vt) {
  const orc_dom* D = &s->d;
  ghost(s, var, vt);
  double Area = 0.0;
  for (int j = 2; j <= D->ny + 1; ++j)
    for (int i = 2; i <= D->nx + 1; ++i) Area = Area + M(D->dxc, i) * M(D->dyc, j);
  for (int k = 1; k <= D->Z; ++k) {
    double rsum = 0.0;
    for (int j = 2; j <= D->ny + 1; ++j)
      for (int i = 2; i <= D->nx + 1; ++i) rsum = rsum + A_(var, i, j, k) * M(D->dxc, i) * M(D->dyc, j);
    outm[k - 1] = rsum / Area;
  }
}

/* Fluctuation a - mean(k) on the interior, ghost 'cfluc', squared over
 * the whole array (NSsolver.F90:316-352, 364-393). */
static void fluct_sq(orc_ns* s, const double* a, const double* mean, double* out) {
  const orc_dom* D = &s->d;
  memcpy(out, a, sizeof(double) * D->G);
  for (int k = 2; k <= D->nz + 1; ++k)
    for (int j = 2; j <= D->ny + 1; ++j)
      for (int i = 2; i <= D->nx + 1; ++i) A_(out, i, j, k) = A_(out, i, j, k) - mean[k - 1];
  ghost(s, out, VT_CFLUC);
  for (long c = 0; c < D->G; ++c) out[c] = out[c] * out[c];
}

/* One pass of the block on the current fields; out = the 16 profiles
 * (Z values each, k = 1..Z): U1, U2, T, S, MKE, TKE, t2, s2 (the *_old
 * arrays after the update), then dU1dt, dU2dt, dTdt, dSdt, dMKEdt, dkdt,
 * dt2dt, ds2dt.  The *_old arrays start at 0.  stretched[d]: axis d uses
 * the interpolation of center_velocity. */
int orc_ns_diagnostics(orc_ns* s, int corrected, const int* stretched, double* out) {
  const orc_dom* D = &s->d;
  const long Z = D->Z, G = D->G;
  for (int d = 0; d < 3; ++d) {
    const int n = d == 0 ? D->nx : (d == 1 ? D->ny : D->nz);
    if (stretched[d] && n < 4) return -1;
  }
  if (!s->dg) {
    s->dg = (double*)calloc(16 * Z, sizeof(double));
    s->dgA = (double*)calloc(G, sizeof(double));
    s->dgB = (double*)calloc(G, sizeof(double));
    s->dgC = (double*)calloc(G, sizeof(double));
    s->dgR = (double*)calloc(G, sizeof(double));
  }
  double* U1o = s->dg;
  double *U2o = U1o + Z, *To = U2o + Z, *So = To + Z, *MKEo = So + Z, *ko = MKEo + Z, *t2o = ko + Z,
         *s2o = t2o + Z;
  double *dU1 = s2o + Z, *dU2 = dU1 + Z, *dT = dU2 + Z, *dS = dT + Z, *dMKE = dS + Z, *dk = dMKE + Z,
         *dt2 = dk + Z, *ds2 = dt2 + Z;
  double* m = (double*)calloc(10 * Z, sizeof(double));
  double *m1 = m, *m2 = m + Z, *m3 = m + 2 * Z, *m4 = m + 3 * Z, *mean = m + 4 * Z, *uu = m + 5 * Z,
         *vv = m + 6 * Z, *ww = m + 7 * Z, *tt = m + 8 * Z, *ss = m + 9 * Z;
  const double dtt = s->time - s->told;
  anel_fields* f = &s->f;
  center_velocity(s, f->u, s->dgA, 1, stretched[0], corrected);
  center_velocity(s, f->v, s->dgB, 2, stretched[1], corrected);
  center_velocity(s, f->w, s->dgC, 3, stretched[2], corrected);
  avg_x1x2(s, s->dgA, m1, VT_U);
  avg_x1x2(s, s->dgB, m2, VT_V);
  avg_x1x2(s, f->rho, m3, VT_RHO);
  avg_x1x2(s, f->scal1, m4, VT_SCAL1);
  for (long k = 0; k < Z; ++k) {
    dU1[k] = (m1[k] - U1o[k]) / dtt;
    U1o[k] = m1[k];
    dU2[k] = (m2[k] - U2o[k]) / dtt;
    U2o[k] = m2[k];
    dT[k] = (m3[k] - To[k]) / dtt;
    To[k] = m3[k];
    dS[k] = (m4[k] - So[k]) / dtt;
    So[k] = m4[k];
    const double tr = m1[k] + m2[k];
    dMKE[k] = (tr - MKEo[k]) / dtt;
    MKEo[k] = tr;
  }
  /* u', v', w' and their squares */
  const int vts[3] = {VT_U, VT_V, VT_W};
  double* cen[3] = {s->dgA, s->dgB, s->dgC};
  double* sq[3] = {uu, vv, ww};
  for (int d = 0; d < 3; ++d) {
    avg_x1x2(s, cen[d], mean, vts[d]);
    fluct_sq(s, cen[d], mean, s->dgR);
    avg_x1x2(s, s->dgR, sq[d], vts[d]);
  }
  for (long k = 0; k < Z; ++k) {
    const double tke = 1.0 / 2.0 * (uu[k] + vv[k] + ww[k]);
    dk[k] = (tke - ko[k]) / dtt;
    ko[k] = tke;
  }
  /* t' and s' */
  avg_x1x2(s, f->rho, mean, VT_RHO);
  fluct_sq(s, f->rho, mean, s->dgR);
  avg_x1x2(s, s->dgR, tt, VT_RHO);
  for (long k = 0; k < Z; ++k) {
    dt2[k] = (tt[k] - t2o[k]) / dtt;
    t2o[k] = tt[k];
  }
  avg_x1x2(s, f->scal1, mean, VT_SCAL1);
  fluct_sq(s, f->scal1, mean, s->dgR);
  avg_x1x2(s, s->dgR, ss, VT_SCAL1);
  for (long k = 0; k < Z; ++k) {
    ds2[k] = (ss[k] - s2o[k]) / dtt;
    s2o[k] = ss[k];
  }
  memcpy(out, s->dg, sizeof(double) * 16 * Z);
  free(m);
  return 0;
}
