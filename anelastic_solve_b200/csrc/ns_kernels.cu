// ns_kernels.cu -- sm_100a kernels of the RK3 sub-step.  Compiled with
// -fmad=false: every sum/product is rounded as the reference's Fortran
// expressions evaluated left to right (citations per kernel).
#include "ns_launch.h"

namespace anel {

static constexpr double R12 = 1.0 / 2.0;  // ratios::r_1_2 (modules.F90:203)
// planes of one (i, j) per thread in the one-cell kernels (SGS, Psource,
// Pgrad): the z-neighbours a thread reads next are the ones it just read
static constexpr int kCellK = 8;

// --------------------------------------------------------------- RHS
// The right-hand-side functions read their fields through an accessor A_:
// FU/FV/FW/FR(i+di, j+dj, k+dk) are u, v, w, rho at a constant offset from
// the cell, FC the scalar of rhs_scalar (rho or scal1), FN/FK the LES
// eddy coefficients (nuT; kappaT for rho, nappaT for scal1).  The accessor
// (TileAcc) reads the shared-memory planes of the tiled kernel or global
// memory around the cell; the floating-point expressions do not depend on
// where the values come from.
#undef FA
#define FU(I, J, K) A_.u((I) - i, (J) - j, (K) - k)
#define FV(I, J, K) A_.v((I) - i, (J) - j, (K) - k)
#define FW(I, J, K) A_.w((I) - i, (J) - j, (K) - k)
#define FR(I, J, K) A_.r((I) - i, (J) - j, (K) - k)
#define FC(I, J, K) (kRho ? A_.r((I) - i, (J) - j, (K) - k) : A_.g(D.s, (I) - i, (J) - j, (K) - k))
#define FN(I, J, K) A_.nu((I) - i, (J) - j, (K) - k)
#define FK(I, J, K) A_.template kap<kRho>(kT, (I) - i, (J) - j, (K) - k)
// r(z) and densityBG(z) at profile index q; with kU (both identically 1,
// the Boussinesq configurations) the constant 1.0, so that products with
// them and quotients by them fold away: x*1 and x/1 are exact, so the
// results are the same bits as with the profile values.
#define RZ(q) (kU ? 1.0 : D.rz[q])
#define BG(q) (kU ? 1.0 : D.bgz[q])

// u1_rhs (NSsolver.F90:646-804): returns Utemp(i,j,k) before ghosting.
template <bool kU, class Acc>
__device__ __forceinline__ double rhs_u(const NSDev& D, const Acc& A_, int i, int j, int k) {
  const double rRe = D.rRe;
  const double rk = RZ(k - 1);
  double acc = 0.0;
  acc = acc +
        rRe * ((FU(i + 1, j, k) - FU(i, j, k)) * MT(D.rdxc, i + 1) -
               (FU(i, j, k) - FU(i - 1, j, k)) * MT(D.rdxc, i)) *
            MT(D.rdxe, i);
  acc = acc +
        rRe * ((FU(i, j + 1, k) - FU(i, j, k)) * MT(D.rdye, j) -
               (FU(i, j, k) - FU(i, j - 1, k)) * MT(D.rdye, j - 1)) *
            MT(D.rdyc, j);
  double ua2 = R12 * (FU(i + 1, j, k) + FU(i, j, k));
  double ua1 = R12 * (FU(i, j, k) + FU(i - 1, j, k));
  acc = acc + (ua1 * ua1 - ua2 * ua2) * MT(D.rdxe, i);
  ua2 = R12 * (FU(i, j, k + 1) + FU(i, j, k));
  ua1 = R12 * (FU(i, j, k) + FU(i, j, k - 1));
  const double ra2 = R12 * (RZ(k) + rk);
  const double ra1 = R12 * (rk + RZ(k - 2));
  const double wa2 = R12 * (FW(i + 1, j, k) + FW(i, j, k));
  const double wa1 = R12 * (FW(i + 1, j, k - 1) + FW(i, j, k - 1));
  acc = acc + (ra1 * ua1 * wa1 - ra2 * ua2 * wa2) * MT(D.rdzc, k) / rk;
  ua2 = R12 * (FU(i, j + 1, k) + FU(i, j, k));
  ua1 = R12 * (FU(i, j, k) + FU(i, j - 1, k));
  const double va2 = R12 * (FV(i + 1, j, k) + FV(i, j, k));
  const double va1 = R12 * (FV(i + 1, j - 1, k) + FV(i, j - 1, k));
  acc = acc + (ua1 * va1 - ua2 * va2) * MT(D.rdyc, j);
  if (D.vles) {  // NSsolver.F90:761-804
    acc = acc - 2.0 *
                    (FN(i + 1, j, k) * (FU(i + 1, j, k) - FU(i, j, k)) * MT(D.rdxc, i + 1) -
                     FN(i, j, k) * (FU(i, j, k) - FU(i - 1, j, k)) * MT(D.rdxc, i)) *
                    MT(D.rdxe, i);
    double n1 = 0.25 * (FN(i, j, k) + FN(i + 1, j, k) + FN(i, j - 1, k) +
                        FN(i + 1, j - 1, k));
    double n2 = 0.25 * (FN(i, j, k) + FN(i + 1, j, k) + FN(i, j + 1, k) +
                        FN(i + 1, j + 1, k));
    acc = acc - 1.0 *
                    (n2 * (FU(i, j + 1, k) - FU(i, j, k)) * MT(D.rdye, j) -
                     n1 * (FU(i, j, k) - FU(i, j - 1, k)) * MT(D.rdye, j - 1)) *
                    MT(D.rdyc, j);
    acc = acc - 1.0 *
                    (n2 * (FV(i + 1, j + 1, k) - FV(i, j + 1, k)) * MT(D.rdxe, i) -
                     n1 * (FV(i + 1, j, k) - FV(i, j, k)) * MT(D.rdxe, i)) *
                    MT(D.rdyc, j);
    n1 = 0.25 * (FN(i, j, k) + FN(i + 1, j, k) + FN(i, j, k - 1) + FN(i + 1, j, k - 1));
    n2 = 0.25 * (FN(i, j, k) + FN(i + 1, j, k) + FN(i, j, k + 1) + FN(i + 1, j, k + 1));
    acc = acc - 1.0 *
                    (ra2 * n2 * (FW(i + 1, j, k) - FW(i, j, k)) * MT(D.rdxe, i) -
                     ra1 * n1 * (FW(i + 1, j, k - 1) - FW(i, j, k - 1)) * MT(D.rdxe, i)) *
                    MT(D.rdzc, k) / rk;
  }
  return acc;
}

// u2_rhs (NSsolver.F90:912-1081)
template <bool kU, class Acc>
__device__ __forceinline__ double rhs_v(const NSDev& D, const Acc& A_, int i, int j, int k) {
  const double rRe = D.rRe;
  const double rk = RZ(k - 1);
  double acc = 0.0;
  acc = acc +
        rRe * ((FV(i + 1, j, k) - FV(i, j, k)) * MT(D.rdxe, i) -
               (FV(i, j, k) - FV(i - 1, j, k)) * MT(D.rdxe, i - 1)) *
            MT(D.rdxc, i);
  acc = acc +
        rRe * ((FV(i, j + 1, k) - FV(i, j, k)) * MT(D.rdyc, j + 1) -
               (FV(i, j, k) - FV(i, j - 1, k)) * MT(D.rdyc, j)) *
            MT(D.rdye, j);
  double va1 = 0.5 * (FV(i, j + 1, k) + FV(i, j, k));
  double va2 = 0.5 * (FV(i, j, k) + FV(i, j - 1, k));
  acc = acc - (va1 * va1 - va2 * va2) * MT(D.rdye, j);
  va1 = 0.5 * (FV(i + 1, j, k) + FV(i, j, k));
  va2 = 0.5 * (FV(i, j, k) + FV(i - 1, j, k));
  const double ua1 = 0.5 * (FU(i, j + 1, k) + FU(i, j, k));
  const double ua2 = 0.5 * (FU(i - 1, j + 1, k) + FU(i - 1, j, k));
  acc = acc - (ua1 * va1 - ua2 * va2) * MT(D.rdxc, i);
  va1 = 0.5 * (FV(i, j, k + 1) + FV(i, j, k));
  va2 = 0.5 * (FV(i, j, k) + FV(i, j, k - 1));
  const double ra1 = 0.5 * (RZ(k) + rk);
  const double ra2 = 0.5 * (rk + RZ(k - 2));
  const double wa1 = 0.5 * (FW(i, j + 1, k) + FW(i, j, k));
  const double wa2 = 0.5 * (FW(i, j + 1, k - 1) + FW(i, j, k - 1));
  acc = acc - (ra1 * wa1 * va1 - ra2 * wa2 * va2) * MT(D.rdzc, k) / rk;
  if (D.vles) {  // NSsolver.F90:1038-1081
    double n1 = 0.25 * (FN(i, j, k) + FN(i - 1, j, k) + FN(i, j + 1, k) +
                        FN(i - 1, j + 1, k));
    double n2 = 0.25 * (FN(i, j, k) + FN(i + 1, j, k) + FN(i, j + 1, k) +
                        FN(i + 1, j + 1, k));
    acc = acc - 1.0 *
                    (n2 * (FV(i + 1, j, k) - FV(i, j, k)) * MT(D.rdxe, i) -
                     n1 * (FV(i, j, k) - FV(i - 1, j, k)) * MT(D.rdxe, i - 1)) *
                    MT(D.rdxc, i);
    acc = acc - 1.0 *
                    (n2 * (FU(i + 1, j + 1, k) - FU(i + 1, j, k)) * MT(D.rdye, j) -
                     n1 * (FU(i, j + 1, k) - FU(i, j, k)) * MT(D.rdye, j)) *
                    MT(D.rdxc, i);
    acc = acc - 2.0 *
                    (FN(i, j + 1, k) * (FV(i, j + 1, k) - FV(i, j, k)) * MT(D.rdyc, j + 1) -
                     FN(i, j, k) * (FV(i, j, k) - FV(i, j - 1, k)) * MT(D.rdyc, j)) *
                    MT(D.rdye, j);
    n1 = 0.25 * (FN(i, j, k) + FN(i, j + 1, k) + FN(i, j, k - 1) + FN(i, j + 1, k - 1));
    n2 = 0.25 * (FN(i, j, k) + FN(i, j + 1, k) + FN(i, j, k + 1) + FN(i, j + 1, k + 1));
    // the reference pairs raver2 (lower face) with nuTaver2 (upper face)
    acc = acc - 1.0 *
                    (ra2 * n2 * (FW(i, j + 1, k) - FW(i, j, k)) * MT(D.rdye, j) -
                     ra1 * n1 * (FW(i, j + 1, k - 1) - FW(i, j, k - 1)) * MT(D.rdye, j)) *
                    MT(D.rdzc, k) / rk;
  }
  return acc;
}

// u3_rhs (NSsolver.F90:1195-1377); rows above nz+1-EW carry no terms.
template <bool kU, class Acc>
__device__ __forceinline__ double rhs_w(const NSDev& D, const Acc& A_, int i, int j, int k) {
  if (k > D.nz + 1 - D.ew) return 0.0;
  const double rRe = D.rRe;
  const double rk = RZ(k - 1), rkp = RZ(k);
  double acc = 0.0;
  acc = acc + R12 * D.g * ((FR(i, j, k + 1) - BG(k)) + (FR(i, j, k) - BG(k - 1))) /
                  (R12 * (BG(k) + BG(k - 1)));
  acc = acc +
        rRe * ((FW(i + 1, j, k) - FW(i, j, k)) * MT(D.rdxe, i) -
               (FW(i, j, k) - FW(i - 1, j, k)) * MT(D.rdxe, i - 1)) *
            MT(D.rdxc, i);
  acc = acc +
        rRe * ((FW(i, j + 1, k) - FW(i, j, k)) * MT(D.rdye, j) -
               (FW(i, j, k) - FW(i, j - 1, k)) * MT(D.rdye, j - 1)) *
            MT(D.rdyc, j);
  double wa1 = 0.5 * (FW(i, j, k + 1) + FW(i, j, k));
  double wa2 = 0.5 * (FW(i, j, k) + FW(i, j, k - 1));
  acc = acc - (rk * wa1 * wa1 - rkp * wa2 * wa2) * MT(D.rdze, k) / (0.5 * (rk + rkp));
  wa1 = 0.5 * (FW(i + 1, j, k) + FW(i, j, k));
  wa2 = 0.5 * (FW(i, j, k) + FW(i - 1, j, k));
  const double ua1 = 0.5 * (FU(i, j, k + 1) + FU(i, j, k));
  const double ua2 = 0.5 * (FU(i - 1, j, k + 1) + FU(i - 1, j, k));
  acc = acc - (ua1 * wa1 - ua2 * wa2) * MT(D.rdxc, i);
  wa1 = 0.5 * (FW(i, j + 1, k) + FW(i, j, k));
  wa2 = 0.5 * (FW(i, j, k) + FW(i, j - 1, k));
  const double va1 = 0.5 * (FV(i, j, k + 1) + FV(i, j, k));
  const double va2 = 0.5 * (FV(i, j - 1, k + 1) + FV(i, j - 1, k));
  acc = acc - (va1 * wa1 - va2 * wa2) * MT(D.rdyc, j);
  if (D.vles) {  // NSsolver.F90:1339-1377
    double n1 = 0.25 * (FN(i, j, k) + FN(i - 1, j, k) + FN(i, j, k + 1) +
                        FN(i - 1, j, k + 1));
    double n2 = 0.25 * (FN(i, j, k) + FN(i + 1, j, k) + FN(i, j, k + 1) +
                        FN(i + 1, j, k + 1));
    acc = acc - 1.0 *
                    (n2 * (FW(i + 1, j, k) - FW(i, j, k)) * MT(D.rdxe, i) -
                     n1 * (FW(i, j, k) - FW(i - 1, j, k)) * MT(D.rdxe, i - 1)) *
                    MT(D.rdxc, i);
    acc = acc - 1.0 *
                    (n2 * (FU(i + 1, j, k + 1) - FU(i + 1, j, k)) * MT(D.rdze, k) -
                     n1 * (FU(i, j, k + 1) - FU(i, j, k)) * MT(D.rdze, k)) *
                    MT(D.rdxc, i);
    n1 = 0.25 * (FN(i, j, k) + FN(i, j - 1, k) + FN(i, j, k + 1) + FN(i, j - 1, k + 1));
    n2 = 0.25 * (FN(i, j, k) + FN(i, j + 1, k) + FN(i, j, k + 1) + FN(i, j + 1, k + 1));
    acc = acc - 1.0 *
                    (n2 * (FW(i, j + 1, k) - FW(i, j, k)) * MT(D.rdye, j) -
                     n1 * (FW(i, j, k) - FW(i, j - 1, k)) * MT(D.rdye, j - 1)) *
                    MT(D.rdyc, j);
    acc = acc - 1.0 *
                    (n2 * (FV(i, j + 1, k + 1) - FV(i, j + 1, k)) * MT(D.rdze, k) -
                     n1 * (FV(i, j, k + 1) - FV(i, j, k)) * MT(D.rdze, k)) *
                    MT(D.rdyc, j);
  }
  return acc;
}

// rho_rhs (NSsolver.F90:1720-1815) and scal1_rhs (:1890-1985)
template <bool kRho, bool kU, class Acc>
__device__ __forceinline__ double rhs_scalar(const NSDev& D, const Acc& A_, int i, int j, int k) {
  const double Dk = kRho ? D.rRe * D.rPr : D.rRe * D.rSc;
  double acc = 0.0;
  acc = acc +
        Dk * ((FC(i + 1, j, k) - FC(i, j, k)) * MT(D.rdxe, i) -
              (FC(i, j, k) - FC(i - 1, j, k)) * MT(D.rdxe, i - 1)) *
            MT(D.rdxc, i);
  acc = acc +
        Dk * ((FC(i, j + 1, k) - FC(i, j, k)) * MT(D.rdye, j) -
              (FC(i, j, k) - FC(i, j - 1, k)) * MT(D.rdye, j - 1)) *
            MT(D.rdyc, j);
  double c2 = 0.5 * (FC(i + 1, j, k) + FC(i, j, k));
  double c1 = 0.5 * (FC(i, j, k) + FC(i - 1, j, k));
  acc = acc + (FU(i - 1, j, k) * c1 - FU(i, j, k) * c2) * MT(D.rdxc, i);
  c2 = 0.5 * (FC(i, j + 1, k) + FC(i, j, k));
  c1 = 0.5 * (FC(i, j, k) + FC(i, j - 1, k));
  acc = acc + (FV(i, j - 1, k) * c1 - FV(i, j, k) * c2) * MT(D.rdyc, j);
  c2 = 0.5 * (FC(i, j, k + 1) + FC(i, j, k));
  c1 = 0.5 * (FC(i, j, k) + FC(i, j, k - 1));
  if (kRho) {
    const double rk = RZ(k - 1);
    const double ra2 = 0.5 * (RZ(k) + rk);
    const double ra1 = 0.5 * (rk + RZ(k - 2));
    acc = acc + (ra1 * FW(i, j, k - 1) * c1 - ra2 * FW(i, j, k) * c2) * MT(D.rdzc, k) / rk;
  } else {
    acc = acc + (FW(i, j, k - 1) * c1 - FW(i, j, k) * c2) * MT(D.rdzc, k);
  }
  if (kRho ? D.rles : D.sles) {
    const double* kT = kRho ? D.kT : D.nT;
    double k2 = 0.5 * (FK(i + 1, j, k) + FK(i, j, k));
    // scal1_rhs keeps the reference's sign slip in the lower average
    double k1 = kRho ? 0.5 * (FK(i, j, k) + FK(i - 1, j, k))
                     : 0.5 * (FK(i, j, k) - FK(i - 1, j, k));
    acc = acc - 1.0 *
                    (k2 * (FC(i + 1, j, k) - FC(i, j, k)) * MT(D.rdxe, i) -
                     k1 * (FC(i, j, k) - FC(i - 1, j, k)) * MT(D.rdxe, i - 1)) *
                    MT(D.rdxc, i);
    k2 = 0.5 * (FK(i, j + 1, k) + FK(i, j, k));
    k1 = kRho ? 0.5 * (FK(i, j, k) + FK(i, j - 1, k))
              : 0.5 * (FK(i, j, k) - FK(i, j - 1, k));
    acc = acc - 1.0 *
                    (k2 * (FC(i, j + 1, k) - FC(i, j, k)) * MT(D.rdye, j) -
                     k1 * (FC(i, j, k) - FC(i, j - 1, k)) * MT(D.rdye, j - 1)) *
                    MT(D.rdyc, j);
  }
  return acc;
}

#undef FA
#define FA(a, i, j, k) (a)[NS_IX(i, j, k)]

// K1: all right-hand sides and the low-storage accumulation
// q = a1*q + a2*F*dt (var_advance, NSsolver.F90:2225-2264) in one pass.
// first = substep with a1 = 0 after zero_temps: q is known to be zero,
// so it is not read (0*0 + x == 0 + x).
//
// Tiled: a block owns 32 (i) x 8 (j) columns and marches kRT_K planes in
// z.  u, v, w and rho are staged in shared memory plane by plane (the
// tile plus a one-cell halo), four planes per field in a ring: the
// functions read planes k-1, k, k+1 while the block brings plane k+2 in
// with asynchronous copies, so every field value is read from global memory once
// per tile instead of once per use.  kL (the eddy coefficients exist):
// nuT and kappaT are staged in the same ring; scal1 and nappaT are read
// from global memory.
constexpr int kRT_I = 32, kRT_J = 8, kRT_K = 32;
constexpr int kRT_W = kRT_I + 2, kRT_PL = kRT_W * (kRT_J + 2);
constexpr int kRT_PER = (kRT_PL + kRT_I * kRT_J - 1) / (kRT_I * kRT_J);  // plane elements per thread

// u, v, w, rho (and with kL nuT and kappaT) from the ring of shared planes
// (slot of plane k = k & 3), the rest from global memory around c0.
template <bool kL>
struct TileAcc {
  const double* sm;  // [field u v w rho (nuT kappaT)][slot][j + 1][i + 1]
  int idx;           // (ty + 1) * kRT_W + tx + 1
  int k;
  const NSDev& D;
  int64_t c0;
  __device__ __forceinline__ double f(int fi, int a, int b, int c) const {
    return sm[(fi * 4 + ((k + c) & 3)) * kRT_PL + idx + b * kRT_W + a];
  }
  __device__ __forceinline__ double u(int a, int b, int c) const { return f(0, a, b, c); }
  __device__ __forceinline__ double v(int a, int b, int c) const { return f(1, a, b, c); }
  __device__ __forceinline__ double w(int a, int b, int c) const { return f(2, a, b, c); }
  __device__ __forceinline__ double r(int a, int b, int c) const { return f(3, a, b, c); }
  __device__ __forceinline__ double g(const double* p, int a, int b, int c) const {
    return p[c0 + a + (int64_t)D.X * b + D.XY * c];
  }
  __device__ __forceinline__ double nu(int a, int b, int c) const {
    return kL ? f(4, a, b, c) : g(D.nuT, a, b, c);
  }
  // p: kappaT for rho (staged with kL), nappaT for scal1 (global)
  template <bool kR>
  __device__ __forceinline__ double kap(const double* p, int a, int b, int c) const {
    return (kL && kR) ? f(5, a, b, c) : g(p, a, b, c);
  }
};

// shared-memory bytes of k_rhs_accum: four planes of 4 (6 with kL) fields
constexpr size_t rhs_smem_bytes(bool les) { return (size_t)(les ? 6 : 4) * 4 * kRT_PL * sizeof(double); }

template <bool kFirst, bool kU, bool kL>
__global__ void __launch_bounds__(kRT_I * kRT_J, 2) k_rhs_accum(NSDev D, double a1, double a2, double dt) {
  extern __shared__ double sm[];
  constexpr int NF = kL ? 6 : 4;
  const int t = threadIdx.x;
  const int tx = t & 31, ty = t >> 5;
  const int i0 = 2 + blockIdx.x * kRT_I, j0 = 2 + blockIdx.y * kRT_J, k0 = 2 + blockIdx.z * kRT_K;
  const int i = i0 + tx, j = j0 + ty;
  const int kend = min(k0 + kRT_K, D.nz + 2);  // exclusive
  const double* fld[6] = {D.u, D.v, D.w, D.rho, D.nuT, D.kT};
  // plane element e of the tile (halo included) -> global offset, or -1
  int64_t off[kRT_PER];
#pragma unroll
  for (int q = 0; q < kRT_PER; ++q) {
    const int e = t + q * kRT_I * kRT_J;
    const int gi = i0 - 1 + e % kRT_W, gj = j0 - 1 + e / kRT_W;
    off[q] = (e < kRT_PL && gi <= D.X && gj <= D.Y) ? NS_IX(gi, gj, 1) : -1;
  }
  // plane p of the four fields into its ring slot, by asynchronous copies
  // (elements outside the array are never read and are skipped)
  auto fetch = [&](int p) {
#pragma unroll
    for (int q = 0; q < kRT_PER; ++q) {
      if (off[q] < 0) continue;
      const int e = t + q * kRT_I * kRT_J;
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const unsigned dst =
            (unsigned)__cvta_generic_to_shared(&sm[(f * 4 + (p & 3)) * kRT_PL + e]);
        const double* src = fld[f] + off[q] + D.XY * (p - 1);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  for (int p = k0 - 1; p <= k0 + 1; ++p) fetch(p);
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  const bool in = i <= D.nx + 1 && j <= D.ny + 1;
  for (int k = k0; k < kend; ++k) {
    const bool pre = k + 1 < kend;  // the next plane's neighbour k+2 is needed
    if (pre) fetch(k + 2);
    if (in) {
      const int64_t c = NS_IX(i, j, k);
      // the accumulators' loads first: their latency overlaps the RHS
      const double q0u = kFirst ? 0.0 : D.qu[c];
      const double q0v = kFirst ? 0.0 : D.qv[c];
      const double q0w = kFirst ? 0.0 : D.qw[c];
      const double q0r = kFirst ? 0.0 : D.qr[c];
      const TileAcc<kL> A{sm, (ty + 1) * kRT_W + tx + 1, k, D, c};
      const double fu = rhs_u<kU>(D, A, i, j, k);
      const double fv = rhs_v<kU>(D, A, i, j, k);
      const double fw = rhs_w<kU>(D, A, i, j, k);
      const double fr = rhs_scalar<true, kU>(D, A, i, j, k);
      D.qu[c] = a1 * q0u + a2 * fu * dt;
      D.qv[c] = a1 * q0v + a2 * fv * dt;
      D.qw[c] = a1 * q0w + a2 * fw * dt;
      D.qr[c] = a1 * q0r + a2 * fr * dt;
      if (D.scal1_on) {
        const double fs = rhs_scalar<false, kU>(D, A, i, j, k);
        const double q0s = kFirst ? 0.0 : D.qs[c];
        D.qs[c] = a1 * q0s + a2 * fs * dt;
      }
    }
    if (pre) asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
  }
}

// ---------------------------------------------------------- ghosting
// bound_update of the two z faces of one column (BC.F90:471-529) after
// the periodic wrap; col(k) = a[base + (k-1)*XY].
__device__ __forceinline__ void zghost_column(const NSDev& D, const ZRule& R, double* a, int64_t base) {
  const int sz = 2, ez = D.nz + 1, iW = R.iw;
  const int64_t XY = D.XY;
#define COL(k) a[base + (int64_t)((k) - 1) * XY]
  auto dzt = [&](int k) { return R.dzt_is_zc ? D.dzc[k - 1] : D.dze[k - 1]; };
  // the serial ghost() first wraps z periodically (BC.F90:64-66)
  COL(sz - 1) = COL(ez);
  COL(ez + 1) = COL(sz);
  for (int face = 1; face <= 2; ++face) {
    const int bt = R.type[face - 1];
    if (R.type[0] == 3 && face == 2) break;  // periodic: bound_update called once
    const double value = R.val[face - 1];
    if (bt == 1) {
      if (face == 1) COL(sz - 1) = value;
      else COL(ez + 1 - iW) = value;
    } else if (bt == 2) {
      if (face == 1) {
        if (R.rt == 1) COL(sz) = COL(sz + 1) - value * dzt(sz + 1 + R.of1);
        COL(sz - 1) = COL(sz) - value * dzt(sz + R.of1);
      } else {
        if (R.rt == 1) COL(ez - iW) = COL(ez - 1 - iW) + value * dzt(ez - 1 + R.of2 - iW);
        COL(ez + 1 - iW) = COL(ez - iW) + value * dzt(ez + R.of2 - iW);
      }
    } else if (bt == 3) {
      COL(sz - 1) = COL(ez - iW);
      COL(ez + 1 - iW) = COL(sz);
    } else if (bt == 4) {
      if (face == 1) COL(sz - 1) = COL(sz) - value * dzt(sz + R.of1);
      else COL(ez + 1 - iW) = COL(ez - iW) + value * dzt(ez + R.of2 - iW);
    } else if (bt == 6) {
      if (face == 1) COL(sz - 1) = 2.0 * value - 1.0 * COL(sz);
      else COL(ez + 1 - iW) = 2.0 * value - 1.0 * COL(ez - iW);
    } else if (bt == 7) {
      if (face == 1) {
        COL(sz) = 0.0;
        COL(sz - 1) = -1.0 * COL(sz + 1);
      } else {
        COL(ez) = 0.0;
        COL(ez + 1 - iW) = -1.0 * COL(ez - iW - 1);
      }
    }
    if (face == 2 && iW == 1) COL(ez + 1) = 0.0;
  }
#undef COL
}

// Periodic images in x and y (BC.F90:55-63 with TB = 3 in x and y) of up
// to three fields, after their interior columns are final (z ghosts
// included): one thread per (ghost column of the ring, k).  Every copy
// reads an interior column, so the order of the copies does not matter:
//   (1, j) <- (nx+1, j), (nx+2, j) <- (2, j)      j = 2..ny+1
//   (i, 1) <- (i, ny+1), (i, ny+2) <- (i, 2)      i = 2..nx+1
//   corners from the diagonally opposite interior column.
struct Fields3 {
  double* a[3];
  int n;
};

__global__ void k_images(NSDev D, Fields3 F) {
  const int nx = D.nx, ny = D.ny;
  const int ring = 2 * ny + 2 * nx + 4;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ring) return;
  const int k = 1 + blockIdx.y;
  int di, dj, si, sj;
  if (t < 2 * ny) {
    const int j = 2 + (t % ny);
    dj = sj = j;
    if (t < ny) {
      di = 1;
      si = nx + 1;
    } else {
      di = nx + 2;
      si = 2;
    }
  } else if (t < 2 * ny + 2 * nx) {
    const int u = t - 2 * ny;
    const int i = 2 + (u % nx);
    di = si = i;
    if (u < nx) {
      dj = 1;
      sj = ny + 1;
    } else {
      dj = ny + 2;
      sj = 2;
    }
  } else {
    const int c = t - 2 * ny - 2 * nx;
    di = (c & 1) ? nx + 2 : 1;
    si = (c & 1) ? 2 : nx + 1;
    dj = (c & 2) ? ny + 2 : 1;
    sj = (c & 2) ? 2 : ny + 1;
  }
  const int64_t dst = NS_IX(di, dj, k), src = NS_IX(si, sj, k);
  for (int f = 0; f < F.n; ++f) F.a[f][dst] = F.a[f][src];
}

// Generic z-ghost pass of one field: one thread per interior column (the
// periodic images follow in k_images).
__global__ void k_ghost_field(NSDev D, double* a, ZRule R) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  if (i > D.nx + 1) return;
  zghost_column(D, R, a, NS_IX(i, j, 1));
}

// ------------------------------------------------------- CN (z implicit)
// var_advance_CN_PL (NSsolver.F90:3054-3465) for one interior column with
// column-independent tridiagonal factors (DNS; r = r(z)).  fac holds, per
// row k = 1..n (n = nz+2): ap (eliminated sub-diagonal), bp (eliminated
// diagonal), c (super-diagonal), t1, t2 (explicit-term weights), rb
// (right-hand side of a wall row) and isbc (1 for wall rows).
struct CNFac {
  const double *ap, *bp, *c, *t1, *t2, *rb, *isbc, *sub, *diag;
};

// The per-row factors and z metrics are staged in shared memory (stride
// n+1 doubles each: ap, bp, c, t1, t2, rb, isbc, rdze, rdzc) and both
// sweeps run in batches of kCNU rows whose global loads are issued before
// any of the batch's stores, so a column costs n/kCNU memory latencies
// instead of n.  The arithmetic and its order are those of the
// row-by-row Thomas algorithm.
constexpr int kCNU = 8;
constexpr int kCNThreads = 256;

// U rows per batch, TPB threads (columns) per block: the launch variants
// the autotuner chooses from (launch_cn); the arithmetic does not depend
// on them.
template <int kVar, int U = kCNU, int TPB = kCNThreads>
__global__ void __launch_bounds__(TPB) k_cn_column(NSDev D, double* __restrict__ fld,
                                                          const double* __restrict__ q, CNFac F,
                                                          double a3, double rkdt, ZRule R) {
  extern __shared__ double cn_sm[];
  const int n = D.nz + 2;
  const int S = n + 1;
  double* s_ap = cn_sm;
  double* s_bp = s_ap + S;
  double* s_c = s_bp + S;
  double* s_t1 = s_c + S;
  double* s_t2 = s_t1 + S;
  double* s_rb = s_t2 + S;
  double* s_bc = s_rb + S;
  double* s_re = s_bc + S;  // rdze
  double* s_rc = s_re + S;  // rdzc
  for (int r = threadIdx.x; r < S; r += blockDim.x) {
    const bool in = r < n;
    s_ap[r] = in ? F.ap[r] : 0.0;
    s_bp[r] = in ? F.bp[r] : 1.0;
    s_c[r] = in ? F.c[r] : 0.0;
    s_t1[r] = in ? F.t1[r] : 0.0;
    s_t2[r] = in ? F.t2[r] : 0.0;
    s_rb[r] = in ? F.rb[r] : 0.0;
    s_bc[r] = in ? F.isbc[r] : 1.0;
    s_re[r] = in ? D.rdze[r] : 0.0;
    s_rc[r] = in ? D.rdzc[r] : 0.0;
  }
  __syncthreads();
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  if (i > D.nx + 1) return;
  const int64_t base = NS_IX(i, j, 1);
  const int64_t XY = D.XY;
  // forward sweep: G(k) = rhs(k) + ap(k) G(k-1); G is stored in place
  double um = fld[base];       // u_old(k-1)
  double uk = fld[base + XY];  // u_old(k)
  double g = s_rb[0];          // row 1 is a wall row
  fld[base] = g;
  for (int kb = 2; kb <= n; kb += U) {
    double up[U], qv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kb + u;
      const int64_t o = base + (int64_t)(k - 1) * XY;
      up[u] = (k < n) ? fld[o + XY] : 0.0;  // u_old(k+1)
      qv[u] = (k <= n) ? q[o] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kb + u;
      if (k <= n) {
        double rhs;
        if (s_bc[k - 1] != 0.0) {
          rhs = s_rb[k - 1];
        } else {
          rhs = 1.0 * uk + a3 * qv[u] * 1.0;
          if (kVar != 3)
            rhs = rhs + rkdt * 0.5 *
                            (s_t2[k - 1] * (up[u] - uk) * s_re[k - 1] -
                             s_t1[k - 1] * (uk - um) * s_re[k - 2]) *
                            s_rc[k - 1];
          else
            rhs = rhs + rkdt * 0.5 *
                            (s_t2[k - 1] * (up[u] - uk) * s_rc[k] -
                             s_t1[k - 1] * (uk - um) * s_rc[k - 1]) *
                            s_re[k - 1];
        }
        g = rhs + s_ap[k - 1] * g;
        fld[base + (int64_t)(k - 1) * XY] = g;
        um = uk;
        uk = up[u];
      }
    }
  }
  // back substitution: G(n) = G(n)/bp(n); G(k) = (G(k) - c(k) G(k+1))/bp(k)
  double gn = g / s_bp[n - 1];
  fld[base + (int64_t)(n - 1) * XY] = gn;
  for (int kb = n - 1; kb >= 1; kb -= U) {
    double gv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kb - u;
      gv[u] = (k >= 1) ? fld[base + (int64_t)(k - 1) * XY] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kb - u;
      if (k >= 1) {
        gn = (gv[u] - s_c[k - 1] * gn) / s_bp[k - 1];
        fld[base + (int64_t)(k - 1) * XY] = gn;
      }
    }
  }
  zghost_column(D, R, fld, base);
}

// LES form of var_advance_CN_PL (NSsolver.F90:3054-3465 with Vmodel =
// SSM): every row adds the eddy terms of the column's kT to the DNS
// coefficients, so the tridiagonal system differs per column and is
// eliminated here (Thomas of mg_relax.F90:541-595: a = -sub/b(k-1),
// b = diag + a c(k-1), G = rhs + a G(k-1)).  G stays in the field and b
// goes to per-cell scratch for the back substitution; the super-diagonal
// c is not stored: the back substitution forms it again from the column's
// kT rows with the same expressions.  Loads of a batch of U rows are
// issued before its stores.  The arithmetic follows the reference's
// expressions term by term.
//
// kU: r is 1 on every plane.  Then ra / rk, and the r-weighted average of
// w's eddy coefficient, leave the coefficient sums unchanged (x * 1.0 and
// x / 1.0 are exact in IEEE arithmetic), so their divisions are left out.

// Eddy weights of row k: t1 (lower face, rows k-1 and k of kT) and t2
// (upper face, rows k and k+1), in the reference's pairing per variable
// (u, v: the four-point average of the two columns; rho: the column's
// two-point average; scal1: the same without r; w: r-weighted).
template <int kVar, bool kU>
__device__ __forceinline__ double les_t1(const double* s_r, int k, double kcc, double knc, double kcm,
                                         double knm) {
  constexpr double H = 0.5;
  if constexpr (kVar == 3) {
    if constexpr (kU) return -kcc;
    const double rk = s_r[k - 1], rkp = s_r[k];
    return -kcc * rk / (H * (rkp + rk));
  } else if constexpr (kVar == 1 || kVar == 2) {
    if constexpr (kU) return -0.25 * (kcc + knc + kcm + knm);
    const double rk = s_r[k - 1];
    const double ra1 = H * (s_r[k] + rk);
    return -0.25 * (kcc + knc + kcm + knm) * ra1 / rk;
  } else if constexpr (kVar == 5) {
    if constexpr (kU) return -0.5 * (kcc + kcm);
    const double rk = s_r[k - 1];
    const double ra1 = H * (s_r[k] + rk);
    return -0.5 * (kcc + kcm) * ra1 / rk;
  } else {
    return -0.5 * (kcc + kcm);
  }
}

template <int kVar, bool kU>
__device__ __forceinline__ double les_t2(const double* s_r, int k, double kcc, double knc, double kcp,
                                         double knp) {
  constexpr double H = 0.5;
  if constexpr (kVar == 3) {
    if constexpr (kU) return -kcp;
    const double rk = s_r[k - 1], rkp = s_r[k];
    return -kcp * rkp / (H * (rkp + rk));
  } else if constexpr (kVar == 1 || kVar == 2) {
    if constexpr (kU) return -0.25 * (kcc + knc + kcp + knp);
    const double rk = s_r[k - 1];
    const double ra2 = H * (rk + s_r[k - 2]);
    return -0.25 * (kcc + knc + kcp + knp) * ra2 / rk;
  } else if constexpr (kVar == 5) {
    if constexpr (kU) return -0.5 * (kcc + kcp);
    const double rk = s_r[k - 1];
    const double ra2 = H * (rk + s_r[k - 2]);
    return -0.5 * (kcc + kcp) * ra2 / rk;
  } else {
    return -0.5 * (kcc + kcp);
  }
}

// super-diagonal of an interior (non-wall) row k from its t2
template <int kVar>
__device__ __forceinline__ double les_sup(const double* s_c, const double* s_re, const double* s_rc, int k,
                                          double rkdt, double t2) {
  if constexpr (kVar != 3)
    return s_c[k - 1] - 0.5 * rkdt * t2 * s_re[k - 1] * s_rc[k - 1];
  else
    return s_c[k - 1] - rkdt * t2 * s_re[k - 1] * s_rc[k];
}

template <int kVar, bool kU, int U = kCNU, int TPB = kCNThreads>
__global__ void __launch_bounds__(TPB) k_cn_column_les(NSDev D, double* __restrict__ fld,
                                                              const double* __restrict__ q, CNFac F,
                                                              double a3, double rkdt, ZRule R,
                                                              const double* __restrict__ kT,
                                                              double* __restrict__ bb) {
  extern __shared__ double cn_sm[];
  const int n = D.nz + 2;
  const int S = n + 1;
  double* s_sub = cn_sm;
  double* s_dia = s_sub + S;
  double* s_c = s_dia + S;
  double* s_t1 = s_c + S;
  double* s_t2 = s_t1 + S;
  double* s_rb = s_t2 + S;
  double* s_bc = s_rb + S;
  double* s_re = s_bc + S;  // rdze
  double* s_rc = s_re + S;  // rdzc
  double* s_r = s_rc + S;   // r(z)
  for (int r = threadIdx.x; r < S; r += blockDim.x) {
    const bool in = r < n;
    s_sub[r] = in ? F.sub[r] : 0.0;
    s_dia[r] = in ? F.diag[r] : 1.0;
    s_c[r] = in ? F.c[r] : 0.0;
    s_t1[r] = in ? F.t1[r] : 0.0;
    s_t2[r] = in ? F.t2[r] : 0.0;
    s_rb[r] = in ? F.rb[r] : 0.0;
    s_bc[r] = in ? F.isbc[r] : 1.0;
    s_re[r] = in ? D.rdze[r] : 0.0;
    s_rc[r] = in ? D.rdzc[r] : 0.0;
    s_r[r] = in ? D.rz[r] : 1.0;
  }
  __syncthreads();
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  if (i > D.nx + 1) return;
  const int64_t base = NS_IX(i, j, 1);
  const int64_t XY = D.XY;
  // eddy coefficient columns: u pairs (i, i+1), v pairs (j, j+1)
  const double* kc = kT + base;
  const double* kn = kT + base + (kVar == 1 ? 1 : (kVar == 2 ? D.X : 0));
  double um = fld[base];
  double uk = fld[base + XY];
  // row 1 is a wall row
  double g = s_rb[0];
  double b = s_dia[0];
  double cprev = s_c[0];
  fld[base] = g;
  bb[base] = b;
  // kT window: rows k-1 and k of both columns (kn = kc for rho, scal1, w)
  double kcm = kc[0], kcc = kc[XY], knm = kn[0], knc = kn[XY];
  for (int kb = 2; kb <= n; kb += U) {
    double up[U], qv[U], kcp[U], knp[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kb + u;
      const int64_t o = (int64_t)(k - 1) * XY;
      up[u] = (k < n) ? fld[base + o + XY] : 0.0;
      qv[u] = (k <= n) ? q[base + o] : 0.0;
      kcp[u] = (k < n) ? kc[o + XY] : 0.0;
      knp[u] = (k < n) ? kn[o + XY] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kb + u;
      if (k <= n) {
        double sub, dia, sup, rhs;
        if (s_bc[k - 1] != 0.0) {
          sub = s_sub[k - 1];
          dia = s_dia[k - 1];
          sup = s_c[k - 1];
          rhs = s_rb[k - 1];
        } else {
          rhs = 1.0 * uk + a3 * qv[u] * 1.0;
          const double t1 = les_t1<kVar, kU>(s_r, k, kcc, knc, kcm, knm);
          const double t2 = les_t2<kVar, kU>(s_r, k, kcc, knc, kcp[u], knp[u]);
          sup = les_sup<kVar>(s_c, s_re, s_rc, k, rkdt, t2);
          if (kVar != 3) {
            rhs = rhs + rkdt * 0.5 *
                            (s_t2[k - 1] * (up[u] - uk) * s_re[k - 1] -
                             s_t1[k - 1] * (uk - um) * s_re[k - 2]) *
                            s_rc[k - 1];
            sub = s_sub[k - 1] - 0.5 * rkdt * t1 * s_re[k - 2] * s_rc[k - 1];
            dia = s_dia[k - 1] + 0.5 * rkdt * (t1 * s_re[k - 2] + t2 * s_re[k - 1]) * s_rc[k - 1];
            rhs = rhs + rkdt * 0.5 *
                            (t2 * (up[u] - uk) * s_re[k - 1] - t1 * (uk - um) * s_re[k - 2]) *
                            s_rc[k - 1];
          } else {
            rhs = rhs + rkdt * 0.5 *
                            (s_t2[k - 1] * (up[u] - uk) * s_rc[k] -
                             s_t1[k - 1] * (uk - um) * s_rc[k - 1]) *
                            s_re[k - 1];
            sub = s_sub[k - 1] - rkdt * t1 * s_re[k - 1] * s_rc[k - 1];
            dia = s_dia[k - 1] + rkdt * (t1 * s_rc[k - 1] + t2 * s_rc[k]) * s_re[k - 1];
            rhs = rhs + rkdt * (t2 * (up[u] - uk) * s_rc[k] - t1 * (uk - um) * s_rc[k - 1]) * s_re[k - 1];
          }
        }
        const double a = -sub / b;
        b = dia + a * cprev;
        g = rhs + a * g;
        const int64_t o = base + (int64_t)(k - 1) * XY;
        fld[o] = g;
        bb[o] = b;
        cprev = sup;
        um = uk;
        uk = up[u];
        kcm = kcc;
        kcc = kcp[u];
        knm = knc;
        knc = knp[u];
      }
    }
  }
  // back substitution: G(n) = G(n)/b(n); G(k) = (G(k) - c(k) G(k+1))/b(k),
  // with c(k) formed again from kT rows k and k+1 (row 1 and the wall rows
  // take the DNS super-diagonal, as in the forward sweep)
  double x = g / b;
  fld[base + (int64_t)(n - 1) * XY] = x;
  double kcu = kc[(int64_t)(n - 1) * XY], knu = kn[(int64_t)(n - 1) * XY];  // rows k+1
  for (int kb = n - 1; kb >= 1; kb -= U) {
    double gv[U], bv[U], kcv[U], knv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kb - u;
      const int64_t o = (int64_t)(k - 1) * XY;
      gv[u] = (k >= 1) ? fld[base + o] : 0.0;
      bv[u] = (k >= 1) ? bb[base + o] : 1.0;
      kcv[u] = (k >= 2) ? kc[o] : 0.0;
      knv[u] = (k >= 2) ? kn[o] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kb - u;
      if (k >= 1) {
        double sup;
        if (k == 1 || s_bc[k - 1] != 0.0) {
          sup = s_c[k - 1];
        } else {
          const double t2 = les_t2<kVar, kU>(s_r, k, kcv[u], knv[u], kcu, knu);
          sup = les_sup<kVar>(s_c, s_re, s_rc, k, rkdt, t2);
        }
        x = (gv[u] - sup * x) / bv[u];
        fld[base + (int64_t)(k - 1) * XY] = x;
        kcu = kcv[u];
        knu = knv[u];
      }
    }
  }
  zghost_column(D, R, fld, base);
}

// ------------------------------------------------------------------ SGS
// SGSdiff (straincal.F90:339-414) with straincal's strain magnitude
// (:48-73) on the interior: nuT = -(Csgs + 0) delg^2 |S| + 0 and the same
// with CTsgs (kappaT) and CSsgs (nappaT); x**2.d0 is x*x.
__global__ void __launch_bounds__(128) k_sgs(NSDev D) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  const int k0 = 2 + blockIdx.z * kCellK;
  if (i > D.nx + 1) return;
  const int kend = min(k0 + kCellK, D.nz + 2);  // exclusive
  for (int k = k0; k < kend; ++k) {
    const double modS = strain_mag(D, D.u, D.v, D.w, i, j, k);
    const double dg2 = D.delg2[k - 1];
    FA(D.nuT, i, j, k) = -(D.Cs[k - 1] + 0.0) * dg2 * modS + 0.0;
    FA(D.kT, i, j, k) = -(D.CTs[k - 1] + 0.0) * dg2 * modS + 0.0;
    FA(D.nT, i, j, k) = -(D.CSs[k - 1] + 0.0) * dg2 * modS + 0.0;
  }
}

// Pressure initial guess: p = 2 h1 - h2 on the interior (the multigrid's
// boundary pass rebuilds the ghosts before the first residual).
__global__ void k_extrap(NSDev D, double* __restrict__ p, const double* __restrict__ h1,
                         const double* __restrict__ h2) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  const int k = 2 + blockIdx.z;
  if (i > D.nx + 1) return;
  FA(p, i, j, k) = 2.0 * FA(h1, i, j, k) - FA(h2, i, j, k);
}

// ------------------------------------------------------------ clipVS
// Routines.F90:301-380 on the interior: below vmin -> vmin, then above
// vmax -> vmax (NaN passes unchanged, as both comparisons are false).
__global__ void k_clip(NSDev D, double* a, double vmin, double vmax) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  const int k = 2 + blockIdx.z;
  if (i > D.nx + 1) return;
  double v = FA(a, i, j, k);
  if (v < vmin) v = vmin;
  if (v > vmax) v = vmax;
  FA(a, i, j, k) = v;
}

// ------------------------------------------------------------ Psource
// NSsolver.F90:2167-2223 (its ghost pass is not needed: the multigrid
// reads the interior of the right-hand side only).
__global__ void k_psource(NSDev D, double rdt) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  const int k0 = 2 + blockIdx.z * kCellK;
  if (i > D.nx + 1) return;
  const int kend = min(k0 + kCellK, D.nz + 2);  // exclusive
  for (int k = k0; k < kend; ++k) {
    const double rk = D.rz[k - 1];
    const double H = 0.5;
    const double v = ((rk * FA(D.u, i, j, k) - rk * FA(D.u, i - 1, j, k)) * MT(D.rdxc, i) +
                      (rk * FA(D.v, i, j, k) - rk * FA(D.v, i, j - 1, k)) * MT(D.rdyc, j) +
                      (H * (D.rz[k] + rk) * FA(D.w, i, j, k) - H * (rk + D.rz[k - 2]) * FA(D.w, i, j, k - 1)) *
                          MT(D.rdzc, k)) *
                     rdt;
    FA(D.psrc, i, j, k) = 0.0 + v;
  }
}

// ------------------------------------------------------ Pgrad + ghosts
// Pgrad (NSsolver.F90:2023-2085): one thread per interior cell (the update
// of a cell reads p only), then ghost(u,'u'), ghost(v,'v'), ghost(w,'w')
// (NSsolver.F90:572-574) by columns.
// hist (may be null): the interior of p is also copied there (the history
// of the pressure initial guess).  kU: r is 1 on every plane, so the
// divisions by r are left out (x / 1.0 == x exactly in IEEE arithmetic).
template <bool kU>
__global__ void __launch_bounds__(128) k_pgrad(NSDev D, double dt, double* __restrict__ hist) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  const int k0 = 2 + blockIdx.z * kCellK;
  if (i > D.nx + 1) return;
  const int kend = min(k0 + kCellK, D.nz + 2);  // exclusive
  const int kend_w = D.nz + 1 - D.ew;
  const double* __restrict__ p = D.p;
  for (int k = k0; k < kend; ++k) {
    const double rk = kU ? 1.0 : D.rz[k - 1];
    const double pk = FA(p, i, j, k);
    if (hist) FA(hist, i, j, k) = pk;
    const double pr = kU ? pk : pk / rk;
    const double pe = kU ? FA(p, i + 1, j, k) : FA(p, i + 1, j, k) / rk;
    const double pn = kU ? FA(p, i, j + 1, k) : FA(p, i, j + 1, k) / rk;
    FA(D.u, i, j, k) = FA(D.u, i, j, k) - (pe - pr) * MT(D.rdxe, i) * dt;
    FA(D.v, i, j, k) = FA(D.v, i, j, k) - (pn - pr) * MT(D.rdye, j) * dt;
    if (k <= kend_w) {
      const double pt = kU ? FA(p, i, j, k + 1) : FA(p, i, j, k + 1) / D.rz[k];
      FA(D.w, i, j, k) = FA(D.w, i, j, k) - (pt - pr) * MT(D.rdze, k) * dt;
    }
  }
}

__global__ void k_pgrad_ghost(NSDev D, ZRule Ru, ZRule Rv, ZRule Rw) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  if (i > D.nx + 1) return;
  const int64_t base = NS_IX(i, j, 1);
  zghost_column(D, Ru, D.u, base);
  zghost_column(D, Rv, D.v, base);
  zghost_column(D, Rw, D.w, base);
}

// -------------------------------------------------------------- calcdt
// Routines.F90:221-233: max over the interior of the advective CFL rate
// (order x, z, y as in the reference), exact integer max of the bits.
__global__ void __launch_bounds__(256) k_cfl_max(NSDev D, unsigned long long* out) {
  // grid-stride over the interior; the maximum of non-negative doubles is
  // taken on their bit patterns, so the result is exact in any order
  __shared__ unsigned long long sh[8];
  const int64_t nx = D.nx, nxy = (int64_t)D.nx * D.ny;
  const int64_t n = nxy * D.nz;
  unsigned long long m = 0;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int k = 2 + (int)(q / nxy);
    const int64_t r = q - (int64_t)(k - 2) * nxy;
    const int j = 2 + (int)(r / nx);
    const int i = 2 + (int)(r - (int64_t)(j - 2) * nx);
    const double adv = MT(D.rdxc, i) * fabs(0.5 * (FA(D.u, i, j, k) + FA(D.u, i - 1, j, k))) +
                       MT(D.rdzc, k) * fabs(0.5 * (FA(D.w, i, j, k) + FA(D.w, i, j, k - 1))) +
                       MT(D.rdyc, j) * fabs(0.5 * (FA(D.v, i, j, k) + FA(D.v, i, j - 1, k)));
    const unsigned long long b = __double_as_longlong(adv);
    m = b > m ? b : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, m, o);
    m = w > m ? w : m;
  }
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) m = sh[q] > m ? sh[q] : m;
    atomicMax(out, m);
  }
}

// divergence (Routines.F90:121-146): max |div| (exact) and the
// volume-weighted sums of |div| and volume (block partials, fixed order)
// divergence() (Routines.F90:54-183): kDivRows consecutive z-cells per
// thread (w of the cell below kept from the previous row), per-block sums
// of |div|*vol and vol in a fixed order, and one atomic maximum per block
// on the bit pattern of max |div| (exact in any order).
constexpr int kDivRows = 8;
// With cfl non-null the same pass also takes calcdt's maximum of
// rdxc |ū| + rdzc |w̄| + rdyc |v̄| (the expression of k_cfl_max, in its
// order) over the same cells and neighbours, for the next step's time
// step: one read of u, v, w at the end of a step serves both.
__global__ void __launch_bounds__(128) k_divergence(NSDev D, unsigned long long* mx, double* part,
                                                    unsigned long long* cfl) {
  __shared__ double sh[2][4];
  __shared__ unsigned long long shm[2][4];
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  const int k0 = 2 + blockIdx.z * kDivRows;
  double s1 = 0.0, s2 = 0.0;
  unsigned long long m = 0, mc = 0;
  if (i <= D.nx + 1) {
    double wb = FA(D.w, i, j, k0 - 1);
    for (int k = k0; k < k0 + kDivRows && k <= D.nz + 1; ++k) {
      const double wt = FA(D.w, i, j, k);
      const double ui = FA(D.u, i, j, k), um = FA(D.u, i - 1, j, k);
      const double vj = FA(D.v, i, j, k), vm = FA(D.v, i, j - 1, k);
      const double d = (ui - um) * MT(D.rdxc, i) + (vj - vm) * MT(D.rdyc, j) + (wt - wb) * MT(D.rdzc, k);
      const double vol = 1.0 / (MT(D.rdxc, i) * MT(D.rdyc, j) * MT(D.rdzc, k));
      s1 += fabs(d) * vol;
      s2 += vol;
      const unsigned long long a = __double_as_longlong(fabs(d));
      m = a > m ? a : m;
      if (cfl) {
        const double adv = MT(D.rdxc, i) * fabs(0.5 * (ui + um)) + MT(D.rdzc, k) * fabs(0.5 * (wt + wb)) +
                           MT(D.rdyc, j) * fabs(0.5 * (vj + vm));
        const unsigned long long b = __double_as_longlong(adv);
        mc = b > mc ? b : mc;
      }
      wb = wt;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, m, o);
    m = w > m ? w : m;
    const unsigned long long wc = __shfl_xor_sync(0xffffffffu, mc, o);
    mc = wc > mc ? wc : mc;
  }
  const int wid = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    sh[0][wid] = s1;
    sh[1][wid] = s2;
    shm[0][wid] = m;
    shm[1][wid] = mc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    unsigned long long mm = 0, mmc = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
      a += sh[0][q];
      b += sh[1][q];
      mm = shm[0][q] > mm ? shm[0][q] : mm;
      mmc = shm[1][q] > mmc ? shm[1][q] : mmc;
    }
    atomicMax(mx, mm);
    if (cfl) atomicMax(cfl, mmc);
    const int64_t bid = blockIdx.x + (int64_t)gridDim.x * (blockIdx.y + (int64_t)gridDim.y * blockIdx.z);
    part[2 * bid] = a;
    part[2 * bid + 1] = b;
  }
}

// ------------------------------------------------------------ launchers
static void launch_images(const NSDev& D, double* a0, double* a1, double* a2, cudaStream_t s) {
  Fields3 F{{a0, a1, a2}, a2 ? 3 : (a1 ? 2 : 1)};
  const int ring = 2 * D.ny + 2 * D.nx + 4;
  k_images<<<dim3((unsigned)((ring + 127) / 128), (unsigned)D.Z, 1u), 128, 0, s>>>(D, F);
  count_launch();
}

static dim3 cell_grid(const NSDev& D, int tx) {
  return dim3((unsigned)((D.nx + tx - 1) / tx), (unsigned)D.ny, (unsigned)D.nz);
}
// kernels whose thread does kCellK planes of one (i, j)
static dim3 cell_grid_k(const NSDev& D, int tx) {
  return dim3((unsigned)((D.nx + tx - 1) / tx), (unsigned)D.ny, (unsigned)((D.nz + kCellK - 1) / kCellK));
}
static dim3 col_grid(const NSDev& D, int tx) {
  return dim3((unsigned)((D.nx + tx - 1) / tx), (unsigned)D.ny, 1u);
}

template <bool kFirst, bool kU, bool kL>
static void rhs_launch(const NSDev& D, dim3 g, double a1, double a2, double dt, cudaStream_t s) {
  const size_t sm = rhs_smem_bytes(kL);
  if (kL) set_smem_limit_once((const void*)k_rhs_accum<kFirst, kU, kL>, (int)sm);
  k_rhs_accum<kFirst, kU, kL><<<g, kRT_I * kRT_J, sm, s>>>(D, a1, a2, dt);
}

void launch_rhs_accum(const NSDev& D, double a1, double a2, double dt, bool first, cudaStream_t s) {
  const dim3 g((unsigned)((D.nx + kRT_I - 1) / kRT_I), (unsigned)((D.ny + kRT_J - 1) / kRT_J),
               (unsigned)((D.nz + kRT_K - 1) / kRT_K));
  const bool les = D.nuT && D.kT;
  const int sel = (first ? 4 : 0) + (D.unit_r ? 2 : 0) + (les ? 1 : 0);
  switch (sel) {
    case 0: rhs_launch<false, false, false>(D, g, a1, a2, dt, s); break;
    case 1: rhs_launch<false, false, true>(D, g, a1, a2, dt, s); break;
    case 2: rhs_launch<false, true, false>(D, g, a1, a2, dt, s); break;
    case 3: rhs_launch<false, true, true>(D, g, a1, a2, dt, s); break;
    case 4: rhs_launch<true, false, false>(D, g, a1, a2, dt, s); break;
    case 5: rhs_launch<true, false, true>(D, g, a1, a2, dt, s); break;
    case 6: rhs_launch<true, true, false>(D, g, a1, a2, dt, s); break;
    default: rhs_launch<true, true, true>(D, g, a1, a2, dt, s); break;
  }
  count_launch();
}

template <int kVar, int U, int TPB>
static void cn_launch(const NSDev& D, double* fld, const double* q, const CNFac& f, double a3, double rkdt,
                      const ZRule& R, cudaStream_t s) {
  const size_t sm = 9 * (size_t)(D.nz + 3) * sizeof(double);
  set_smem_limit_once((const void*)k_cn_column<kVar, U, TPB>, 200 * 1024);
  k_cn_column<kVar, U, TPB><<<col_grid(D, TPB), TPB, sm, s>>>(D, fld, q, f, a3, rkdt, R);
}

template <int kVar>
static void cn_variant(const NSDev& D, double* fld, const double* q, const CNFac& f, double a3, double rkdt,
                       const ZRule& R, int variant, cudaStream_t s) {
  switch (variant) {
    case 1: cn_launch<kVar, 16, 128>(D, fld, q, f, a3, rkdt, R, s); break;
    case 2: cn_launch<kVar, 16, 256>(D, fld, q, f, a3, rkdt, R, s); break;
    case 3: cn_launch<kVar, 32, 128>(D, fld, q, f, a3, rkdt, R, s); break;
    default: cn_launch<kVar, kCNU, kCNThreads>(D, fld, q, f, a3, rkdt, R, s); break;
  }
}

void launch_cn(const NSDev& D, int var, double* fld, const double* q, const CNFacHost& F, double a3,
               double rkdt, const ZRule& R, int variant, cudaStream_t s) {
  CNFac f{F.ap, F.bp, F.c, F.t1, F.t2, F.rb, F.isbc, F.sub, F.diag};
  if (var == 3) cn_variant<3>(D, fld, q, f, a3, rkdt, R, variant, s);
  else cn_variant<1>(D, fld, q, f, a3, rkdt, R, variant, s);
  count_launch();
  launch_images(D, fld, nullptr, nullptr, s);
}

template <int kVar, int U, int TPB>
static void cn_les_launch(const NSDev& D, double* fld, const double* q, const CNFac& f, double a3, double rkdt,
                          const ZRule& R, const double* kT, double* b, cudaStream_t s) {
  const size_t sm = 10 * (size_t)(D.nz + 3) * sizeof(double);
  if (D.unit_r) {
    set_smem_limit_once((const void*)k_cn_column_les<kVar, true, U, TPB>, 200 * 1024);
    k_cn_column_les<kVar, true, U, TPB><<<col_grid(D, TPB), TPB, sm, s>>>(D, fld, q, f, a3, rkdt, R, kT, b);
  } else {
    set_smem_limit_once((const void*)k_cn_column_les<kVar, false, U, TPB>, 200 * 1024);
    k_cn_column_les<kVar, false, U, TPB><<<col_grid(D, TPB), TPB, sm, s>>>(D, fld, q, f, a3, rkdt, R, kT, b);
  }
}

template <int kVar>
static void cn_les_variant(const NSDev& D, double* fld, const double* q, const CNFac& f, double a3, double rkdt,
                           const ZRule& R, const double* kT, double* b, int variant, cudaStream_t s) {
  switch (variant) {
    case 1: cn_les_launch<kVar, 4, 128>(D, fld, q, f, a3, rkdt, R, kT, b, s); break;
    case 2: cn_les_launch<kVar, 8, 128>(D, fld, q, f, a3, rkdt, R, kT, b, s); break;
    case 3: cn_les_launch<kVar, 16, 128>(D, fld, q, f, a3, rkdt, R, kT, b, s); break;
    default: cn_les_launch<kVar, kCNU, kCNThreads>(D, fld, q, f, a3, rkdt, R, kT, b, s); break;
  }
}

void launch_cn_les(const NSDev& D, int var, double* fld, const double* q, const CNFacHost& F, double a3,
                   double rkdt, const ZRule& R, const double* kT, double* b, int variant, cudaStream_t s) {
  CNFac f{F.ap, F.bp, F.c, F.t1, F.t2, F.rb, F.isbc, F.sub, F.diag};
  switch (var) {
    case 1: cn_les_variant<1>(D, fld, q, f, a3, rkdt, R, kT, b, variant, s); break;
    case 2: cn_les_variant<2>(D, fld, q, f, a3, rkdt, R, kT, b, variant, s); break;
    case 3: cn_les_variant<3>(D, fld, q, f, a3, rkdt, R, kT, b, variant, s); break;
    case 5: cn_les_variant<5>(D, fld, q, f, a3, rkdt, R, kT, b, variant, s); break;
    default: cn_les_variant<8>(D, fld, q, f, a3, rkdt, R, kT, b, variant, s); break;
  }
  count_launch();
  launch_images(D, fld, nullptr, nullptr, s);
}

void launch_sgs(const NSDev& D, const ZRule& cfluc, cudaStream_t s) {
  k_sgs<<<cell_grid_k(D, 128), 128, 0, s>>>(D);
  for (double* a : {D.nuT, D.kT, D.nT}) k_ghost_field<<<col_grid(D, 64), 64, 0, s>>>(D, a, cfluc);
  count_launch(4);
  launch_images(D, D.nuT, D.kT, D.nT, s);
}

// ------------------------------------------------------ plane statistics
// The driver's per-step dk/dt block (NSsolver.F90:288-395).

// Newton form through five points (divdiffs + interpoly,
// StatTools.F90:563-653) of y over the abscissae x, evaluated at loc.
__device__ __forceinline__ double newton5(const double (&x)[5], const double (&y)[5], double loc) {
  double Dm[5][5];
#pragma unroll
  for (int k = 0; k <= 4; ++k) Dm[k][0] = y[k];
#pragma unroll
  for (int j = 1; j <= 4; ++j)
#pragma unroll
    for (int k = j; k <= 4; ++k) Dm[k][j] = (Dm[k][j - 1] - Dm[k - 1][j - 1]) / (x[k] - x[k - j]);
  double sum1 = Dm[4][4];
#pragma unroll
  for (int k = 3; k >= 0; --k) sum1 = sum1 * (loc - x[k]) + Dm[k][k];
  return sum1;
}

// center_velocity (StatTools.F90:87-289) of the component staggered in
// direction dir, interior cells: the mean of the two faces on a uniform
// axis; on a stretched one interpoly(dep, ind, loc, 4) over the window
// q-2..q+2 (sx-1..sx+3 at sx, ex-3..ex+1 at ex).  As written (corrected =
// 0) interpoly hands the values to divdiffs as the abscissae; corrected
// interpolates the values over the coordinates.  e, c: the edge and
// centre coordinates of the axis.
__global__ void k_center(NSDev D, const double* __restrict__ in, double* __restrict__ out, int dir,
                         int stretched, int corrected, const double* __restrict__ e,
                         const double* __restrict__ c) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  const int k = 2 + blockIdx.z;
  if (i > D.nx + 1) return;
  const int64_t o = NS_IX(i, j, k);
  const int64_t st = dir == 1 ? 1 : (dir == 2 ? (int64_t)D.X : D.XY);
  if (!stretched) {
    out[o] = R12 * (in[o] + in[o - st]);
    return;
  }
  const int q = dir == 1 ? i : (dir == 2 ? j : k);
  const int n = dir == 1 ? D.nx : (dir == 2 ? D.ny : D.nz);
  const int lo = q == 2 ? 1 : (q == n + 1 ? n - 2 : q - 2);
  double dep[5], ind[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    dep[m] = in[o + (int64_t)(lo + m - q) * st];
    ind[m] = e[lo + m - 1];
  }
  out[o] = corrected ? newton5(ind, dep, c[q - 1]) : newton5(dep, ind, c[q - 1]);
}

// Squared fluctuation (a - mean(k))^2 on the interior (NSsolver.F90:316-
// 352, 364-393); the ghost pass of the field's rule that follows rebuilds
// every ghost cell from the interior, as avgX1X2's ghost call does.
__global__ void k_fluct_sq(NSDev D, const double* __restrict__ a, const double* __restrict__ mean,
                           double* __restrict__ out) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  const int k = 2 + blockIdx.z;
  if (i > D.nx + 1) return;
  const int64_t o = NS_IX(i, j, k);
  const double t = a[o] - mean[k - 1];
  out[o] = t * t;
}

// avgX1X2 (Average.F90:279-368) for cell-centred types: per plane k = 1..Z
// the sum of a(i,j,k)*dxc(i)*dyc(j) over the interior (i,j), as
// kPlaneBlocks partial sums per plane (block b takes rows j = 2+b, 2+b+B,
// ...), then a fixed-order fold divided by Area.  Deterministic for a
// given grid; the order differs from the reference's single running sum.
constexpr int kPlaneBlocks = 32;
constexpr int kPlaneThreads = 256;
__global__ void __launch_bounds__(kPlaneThreads) k_plane_part(NSDev D, const double* __restrict__ a,
                                                             const double* __restrict__ wx,
                                                             const double* __restrict__ wy,
                                                             double* __restrict__ part) {
  __shared__ double sh[kPlaneThreads / 32];
  const int k = 1 + blockIdx.y;
  double acc = 0.0;
  for (int j = 2 + blockIdx.x; j <= D.ny + 1; j += gridDim.x) {
    const double wyj = wy[j - 1];
    const int64_t base = NS_IX(0, j, k);
    for (int i = 2 + threadIdx.x; i <= D.nx + 1; i += blockDim.x) acc += a[base + i] * wx[i - 1] * wyj;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kPlaneThreads / 32; ++w) t += sh[w];
    part[(int64_t)(k - 1) * gridDim.x + blockIdx.x] = t;
  }
}

__global__ void k_plane_fold(int Z, int nb, const double* __restrict__ part, double area,
                             double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= Z) return;
  double t = 0.0;
  for (int b = 0; b < nb; ++b) t += part[(int64_t)k * nb + b];
  out[k] = t / area;
}

// The profile bookkeeping of the block: m = plane means (uc, vc, rho,
// scal1, wc) then second moments (u'u', v'v', w'w', t't', s's'), Z each;
// dg = U1, U2, T, S, MKE, TKE, t2, s2 (previous values in, new out), then
// their derivatives (new - old) / dtt.
__global__ void k_diag_update(int Z, double dtt, const double* __restrict__ m, double* __restrict__ dg) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= Z) return;
  const double m1 = m[k], m2 = m[Z + k], m3 = m[2 * Z + k], m4 = m[3 * Z + k];
  const double uu = m[5 * Z + k], vv = m[6 * Z + k], ww = m[7 * Z + k];
  const double tt = m[8 * Z + k], ss = m[9 * Z + k];
  const double tr = m1 + m2;
  const double tke = 1.0 / 2.0 * (uu + vv + ww);
  const double now[8] = {m1, m2, m3, m4, tr, tke, tt, ss};
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    dg[(8 + q) * Z + k] = (now[q] - dg[q * Z + k]) / dtt;
    dg[q * Z + k] = now[q];
  }
}

void launch_center(const NSDev& D, const double* in, double* out, int dir, int stretched, int corrected,
                   const double* e, const double* c, cudaStream_t s) {
  k_center<<<cell_grid(D, 128), 128, 0, s>>>(D, in, out, dir, stretched, corrected, e, c);
  count_launch();
}

void launch_fluct_sq(const NSDev& D, const double* a, const double* mean, double* out, cudaStream_t s) {
  k_fluct_sq<<<cell_grid(D, 128), 128, 0, s>>>(D, a, mean, out);
  count_launch();
}

int64_t plane_part_doubles(const NSDev& D) { return (int64_t)kPlaneBlocks * D.Z; }

void launch_plane_avg(const NSDev& D, const double* a, const double* wx, const double* wy, double area,
                      double* part, double* out, cudaStream_t s) {
  k_plane_part<<<dim3(kPlaneBlocks, (unsigned)D.Z), kPlaneThreads, 0, s>>>(D, a, wx, wy, part);
  k_plane_fold<<<(D.Z + 127) / 128, 128, 0, s>>>(D.Z, kPlaneBlocks, part, area, out);
  count_launch(2);
}

void launch_diag_update(int Z, double dtt, const double* m, double* dg, cudaStream_t s) {
  k_diag_update<<<(Z + 127) / 128, 128, 0, s>>>(Z, dtt, m, dg);
  count_launch();
}

// Park-Miller minimal standard: element n (0-based) of the sequence of a
// seed is seed * 16807^(n+1) mod (2^31-1) (Park & Miller, CACM 31(10),
// 1988); the power by binary exponentiation, products below 2^62.
__device__ __forceinline__ double park_miller_at(uint64_t seed, uint64_t n) {
  const uint64_t m = 2147483647ull;
  uint64_t r = 1, b = 16807ull, e = n + 1;
  while (e) {
    if (e & 1) r = (r * b) % m;
    b = (b * b) % m;
    e >>= 1;
  }
  const uint64_t x = (seed * r) % m;
  return (double)x / 2147483647.0;
}

__global__ void k_init_shear(NSDev D, const double* __restrict__ prof, uint64_t seed, double amp,
                             double zmax) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < D.G;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int k = 1 + (int)(c / D.XY);
    const double th = prof[k - 1];
    const bool in = prof[D.Z + k - 1] < zmax;
    double pert[3];
    for (int q = 0; q < 3; ++q)
      pert[q] = in ? amp * (2.0 * park_miller_at(seed, (uint64_t)q * D.G + c) - 1.0) : 0.0;
    D.u[c] = th + pert[0];
    D.v[c] = 0.0 + pert[1];
    D.w[c] = 0.0 + pert[2];
    D.rho[c] = -th;
    D.p[c] = 0.0;
    D.s[c] = 0.0;
  }
}

void launch_init_shear(const NSDev& D, const double* prof, uint32_t seed, double amp, double zmax,
                       cudaStream_t s) {
  int64_t b = (D.G + 255) / 256;
  if (b > 148 * 8) b = 148 * 8;
  const uint64_t sd = (uint64_t)seed % 2147483647ull;
  k_init_shear<<<(unsigned)b, 256, 0, s>>>(D, prof, sd ? sd : 1ull, amp, zmax);
  count_launch();
}

void launch_clip(const NSDev& D, double* a, double vmin, double vmax, cudaStream_t s) {
  k_clip<<<cell_grid(D, 128), 128, 0, s>>>(D, a, vmin, vmax);
  count_launch();
}

void launch_psource(const NSDev& D, double dt, cudaStream_t s) {
  const int tx = 128;
  k_psource<<<cell_grid_k(D, tx), tx, 0, s>>>(D, 1.0 / dt);
  count_launch();
}

void launch_extrap(const NSDev& D, double* p, const double* h1, const double* h2, cudaStream_t s) {
  k_extrap<<<cell_grid(D, 128), 128, 0, s>>>(D, p, h1, h2);
  count_launch();
}

void launch_pgrad(const NSDev& D, double dt, const ZRule& Ru, const ZRule& Rv, const ZRule& Rw,
                  cudaStream_t s, double* hist) {
  if (D.unit_r)
    k_pgrad<true><<<cell_grid_k(D, 128), 128, 0, s>>>(D, dt, hist);
  else
    k_pgrad<false><<<cell_grid_k(D, 128), 128, 0, s>>>(D, dt, hist);
  k_pgrad_ghost<<<col_grid(D, 64), 64, 0, s>>>(D, Ru, Rv, Rw);
  count_launch(2);
  launch_images(D, D.u, D.v, D.w, s);
}

void launch_ghost_field(const NSDev& D, double* a, const ZRule& R, cudaStream_t s) {
  const int tx = 64;
  k_ghost_field<<<col_grid(D, tx), tx, 0, s>>>(D, a, R);
  count_launch();
  launch_images(D, a, nullptr, nullptr, s);
}

void launch_cfl_max(const NSDev& D, unsigned long long* out, cudaStream_t s) {
  const int64_t cells = (int64_t)D.nx * D.ny * D.nz;
  int64_t blocks = (cells + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_cfl_max<<<(unsigned)blocks, 256, 0, s>>>(D, out);
  count_launch();
}

static dim3 divergence_grid(const NSDev& D) {
  return dim3((unsigned)((D.nx + 127) / 128), (unsigned)D.ny, (unsigned)((D.nz + kDivRows - 1) / kDivRows));
}

int64_t divergence_blocks(const NSDev& D) {
  const dim3 g = divergence_grid(D);
  return (int64_t)g.x * g.y * g.z;
}

void launch_divergence(const NSDev& D, unsigned long long* mx, double* part, cudaStream_t s,
                       unsigned long long* cfl) {
  k_divergence<<<divergence_grid(D), 128, 0, s>>>(D, mx, part, cfl);
  count_launch();
}

}  // namespace anel
