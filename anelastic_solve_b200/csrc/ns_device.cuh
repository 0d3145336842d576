// ns_device.cuh -- device code of the RK3 sub-step (rk_ss of
// ANELASTIC_SL/dns/NSsolver.F90:418-583).  FP64, compiled with
// -fmad=false; every expression is evaluated in the reference's order so
// the fields match the Fortran semantics bit for bit.
//
// Requirements of this implementation (checked on the host): x and y
// periodic for every field, density r and densityBG functions of z only.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace anel {

// field ghost types (the vtype strings of ghost(), BC.F90:67-95)
enum NSVtype { NV_U = 0, NV_V, NV_W, NV_P, NV_RHO, NV_CFLUC, NV_PSOURCE, NV_UTEMP, NV_VTEMP,
               NV_WTEMP, NV_RTEMP, NV_S1TEMP, NV_SCAL1, NV_SCAL1TEMP };

// z-wall rule of one field type: bound_update of both z faces
// (BC.F90:471-529) with the staggering offsets and metric of the type.
struct ZRule {
  int type[2];     // Btype at z-min / z-max (1,2,3,4,6,7)
  double val[2];   // VB
  int rt;          // two-point Neumann
  int iw;          // edge-node shift (EW for w types)
  int of1, of2;    // staggering offsets
  int dzt_is_zc;   // metric: 1 -> dzc, 0 -> dze
};

struct NSDev {
  int nx, ny, nz;
  int X, Y, Z;
  int64_t XY, G;
  // metrics, [idx-1] for the Fortran index
  const double *rdxe, *rdxc, *rdye, *rdyc, *rdze, *rdzc, *dze, *dzc;
  const double *rz, *bgz;  // r(:,:,k), densityBG(:,:,k)
  double *u, *v, *w, *p, *rho, *s;
  double *qu, *qv, *qw, *qr, *qs;
  double* psrc;
  double *nuT, *kT, *nT;
  const double *Cs, *CTs, *CSs, *delg2;  // LES: Csgs, CTsgs, CSsgs, delg**2 profiles (k)
  double rRe, rPr, rSc, g;
  int vles, rles, sles;  // Vmodel / Rmodel / Smodel are SSM
  int ew;
  int scal1_on;
  int unit_r;  // r and densityBG are 1 on every plane (ghosts included)
};

#define NS_IX(i, j, k) ((int64_t)((i) - 1) + (int64_t)D.X * ((j) - 1) + D.XY * ((k) - 1))
#define FA(a, i, j, k) (a)[NS_IX(i, j, k)]
#define MT(a, i) (a)[(i) - 1]

// straincal's strain magnitude (straincal.F90:48-73) of (l1, l2, l3) at an
// interior cell; x**2.d0 is x*x.
__device__ __forceinline__ double strain_mag(const NSDev& D, const double* l1, const double* l2,
                                             const double* l3, int i, int j, int k) {
  const double TS11 = (FA(l1, i + 1, j, k) - FA(l1, i, j, k)) * MT(D.rdxc, i);
  const double TS22 = (FA(l2, i, j + 1, k) - FA(l2, i, j, k)) * MT(D.rdyc, j);
  const double TS33 = (FA(l3, i, j, k + 1) - FA(l3, i, j, k)) * MT(D.rdzc, k);
  double t1 = 0.25 * (FA(l1, i, j, k) + FA(l1, i + 1, j, k) + FA(l1, i, j + 1, k) + FA(l1, i + 1, j + 1, k));
  double t2 = 0.25 * (FA(l1, i, j, k) + FA(l1, i + 1, j, k) + FA(l1, i, j - 1, k) + FA(l1, i + 1, j - 1, k));
  double t3 = 0.25 * (FA(l2, i, j, k) + FA(l2, i, j + 1, k) + FA(l2, i + 1, j, k) + FA(l2, i + 1, j + 1, k));
  double t4 = 0.25 * (FA(l2, i, j, k) + FA(l2, i, j + 1, k) + FA(l2, i - 1, j, k) + FA(l2, i - 1, j + 1, k));
  const double TS12 = 0.5 * ((t1 - t2) * MT(D.rdyc, j) + (t3 - t4) * MT(D.rdxc, i));
  t1 = 0.25 * (FA(l1, i, j, k) + FA(l1, i + 1, j, k) + FA(l1, i, j, k + 1) + FA(l1, i + 1, j, k + 1));
  t2 = 0.25 * (FA(l1, i, j, k) + FA(l1, i + 1, j, k) + FA(l1, i, j, k - 1) + FA(l1, i + 1, j, k - 1));
  t3 = 0.25 * (FA(l3, i, j, k) + FA(l3, i, j, k + 1) + FA(l3, i + 1, j, k) + FA(l3, i + 1, j, k + 1));
  t4 = 0.25 * (FA(l3, i, j, k) + FA(l3, i, j, k + 1) + FA(l3, i - 1, j, k) + FA(l3, i - 1, j, k + 1));
  const double TS13 = 0.5 * ((t1 - t2) * MT(D.rdzc, k) + (t3 - t4) * MT(D.rdxc, i));
  t1 = 0.25 * (FA(l2, i, j, k) + FA(l2, i, j + 1, k) + FA(l2, i, j, k + 1) + FA(l2, i, j + 1, k + 1));
  t2 = 0.25 * (FA(l2, i, j, k) + FA(l2, i, j + 1, k) + FA(l2, i, j, k - 1) + FA(l2, i, j + 1, k - 1));
  t3 = 0.25 * (FA(l3, i, j, k) + FA(l3, i, j, k + 1) + FA(l3, i, j + 1, k) + FA(l3, i, j + 1, k + 1));
  t4 = 0.25 * (FA(l3, i, j, k) + FA(l3, i, j, k + 1) + FA(l3, i, j - 1, k) + FA(l3, i, j - 1, k + 1));
  const double TS23 = 0.5 * ((t1 - t2) * MT(D.rdzc, k) + (t3 - t4) * MT(D.rdyc, j));
  return sqrt(2.0) * sqrt(TS11 * TS11 + TS22 * TS22 + TS33 * TS33 + 2.0 * (TS12 * TS12) + 2.0 * (TS13 * TS13) +
                          2.0 * (TS23 * TS23));
}

}  // namespace anel
