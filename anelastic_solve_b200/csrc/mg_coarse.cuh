// mg_coarse.cuh -- FP64 direct solve of a coarse level of the z-line cycle.
//
// On a level with x and y periodic and x/y-uniform, symmetric line
// coefficients (a1 == a2, a3 == a4), the operator
//   a1 (phi(i-1) + phi(i+1)) + a3 (phi(j-1) + phi(j+1)) + cz5 phi(k-1) + cz6 phi(k+1) + D(k) phi
// is diagonalised in x and y by the real orthonormal Fourier basis
// (constant, cos and sin pairs, the alternating mode for an even count):
// basis function p of x has eigenvalue 2 a1 cos(theta_p) of the x part.  So
// the solve is a transform of every z-plane into modes (two small dense
// products per plane), one tridiagonal z-system per mode (nz = 32*M rows;
// the z-ghost rule of the level folded into the first and last rows), and
// the inverse transform.  A mode's system is solved by one warp as in the
// column sweep (lane s owns rows s*M .. s*M+M-1; inner rows by Thomas
// elimination, the 32 separators by cyclic reduction over the lanes), in
// FP64 with per-mode factors precomputed on the host.  The mode that is
// constant in x and y is singular under Neumann z walls (constant null
// vector): its last row is replaced by phi = 0, which pins the gauge.
//
// In the mixed-precision cycle this replaces the relaxation of the chosen
// level and of every level below it: the FP32 residual restricted to the
// level is solved exactly in FP64 and handed back to the cycle in FP32.
#pragma once

#include "mg_col.cuh"

namespace anel {

constexpr int kDirMaxN = 64;       // largest x or y extent of a directly solved level
constexpr int kDirMaxModes = 512;  // largest nx * ny of a directly solved level

// doubles of one mode's factor block: the column-sweep factors
// (col_fac_floats(M) values, in FP64) and the scale of the last row's
// right-hand side (0 on the pinned mode), padded to 32
__host__ __device__ constexpr int dir_fac_per_mode(int M) { return col_fac_floats(M) + 32; }

struct DirectFac {
  int nx, ny, nz, nm;  // interior extents, nm = nx * ny modes (p + nx*q)
  int M;               // rows per lane, nz = 32*M
  const double* Bx;    // nx x nx, row p = basis function p over i
  const double* By;    // ny x ny
  const double* fac;   // [nm][dir_fac_per_mode(M)]
  double* work;        // [nmem][nm][nz] modal right-hand side, then solution
  // members of a batch (the same level of independent problems): member b
  // has its own work block; act[b] == 0 skips it (null: all active)
  int nmem = 1;
  const int* act = nullptr;
};

// input: the level's restricted FP32 right-hand side (column layout)
struct DirColIn {
  ColLevel L;
  __device__ __forceinline__ DirColIn member(int b) const { return DirColIn{col_member(L, b)}; }
  __device__ __forceinline__ double get(int i0, int j0, int r) const {
    return (double)L.src[col_cell(L, i0 + 2, j0 + 2, r + 2)];
  }
};
// output: the level's FP32 phi (column layout) with its ghost copies
struct DirColOut {
  ColLevel L;
  __device__ __forceinline__ DirColOut member(int b) const { return DirColOut{col_member(L, b)}; }
  __device__ __forceinline__ void put(int i0, int j0, int r, double v) const {
    const int i = i0 + 2, j = j0 + 2, k = r + 2;
    const float f = (float)v;
    int d0 = kNoImage, d1 = kNoImage, d2 = kNoImage;
    if (L.img) {
      const int* im = L.img + 3 * (i0 + (int64_t)L.nx * j0);
      d0 = im[0];
      d1 = im[1];
      d2 = im[2];
    }
    const bool h0 = d0 != kNoImage, h1 = d1 != kNoImage, h2 = d2 != kNoImage;
    const int64_t o0 = (int64_t)d0 * L.CS, o1 = (int64_t)d1 * L.CS, o2 = (int64_t)d2 * L.CS;
    const int64_t c = col_cell(L, i, j, k);
    float* P = L.phi;
    col_put(P, c, f, o0, o1, o2, h0, h1, h2);
    const int64_t g1 = c - (k - 1), gZ = c + (L.nz + 2 - k);
    if (r == 0) {
      if (L.z1 != 2) col_put(P, g1, L.z1 == 1 ? f : 0.f, o0, o1, o2, h0, h1, h2);
      if (L.zZ != 2) col_put(P, gZ, L.zZ == 1 ? f : 0.f, o0, o1, o2, h0, h1, h2);
    }
    if (r == L.nz - 1) {
      if (L.z1 == 2) col_put(P, g1, f, o0, o1, o2, h0, h1, h2);
      if (L.zZ == 2) col_put(P, gZ, f, o0, o1, o2, h0, h1, h2);
    }
  }
};
// FP64 reference layout (interior only; the caller runs the boundary pass)
struct DirRowIn {
  const double* f;
  int X;
  int64_t XY;
  __device__ __forceinline__ DirRowIn member(int) const { return *this; }
  __device__ __forceinline__ double get(int i0, int j0, int r) const {
    return f[cidx(i0 + 2, j0 + 2, r + 2, X, XY)];
  }
};
struct DirRowOut {
  double* phi;
  int X;
  int64_t XY;
  __device__ __forceinline__ DirRowOut member(int) const { return *this; }
  __device__ __forceinline__ void put(int i0, int j0, int r, double v) const {
    phi[cidx(i0 + 2, j0 + 2, r + 2, X, XY)] = v;
  }
};

// One CTA per z-row of a member: W = Bx F By^T of the row's plane.
template <class In>
__global__ void __launch_bounds__(256) k_dir_forward(DirectFac F, In inb) {
  extern __shared__ double dsm[];
  const int b = blockIdx.x / F.nz;
  if (F.act && !F.act[b]) return;  // the whole CTA
  const In in = inb.member(b);
  double* work = F.work + (int64_t)b * F.nm * F.nz;
  const int nx = F.nx, ny = F.ny, r = blockIdx.x - b * F.nz;
  double* bx = dsm;
  double* by = bx + nx * nx;
  double* P = by + ny * ny;
  double* T = P + nx * ny;
  // Bx transposed (bx[i*nx + p]): the lanes of a warp take consecutive p
  // below and read consecutive words instead of one bank nx words apart
  for (int q = threadIdx.x; q < nx * nx; q += blockDim.x) bx[(q % nx) * nx + q / nx] = F.Bx[q];
  for (int q = threadIdx.x; q < ny * ny; q += blockDim.x) by[q] = F.By[q];
  for (int q = threadIdx.x; q < nx * ny; q += blockDim.x) P[q] = in.get(q % nx, q / nx, r);
  __syncthreads();
  for (int q = threadIdx.x; q < nx * ny; q += blockDim.x) {  // T(p, j)
    const int p = q % nx, j = q / nx;
    double s = 0.0;
    for (int i = 0; i < nx; ++i) s += bx[i * nx + p] * P[i + nx * j];
    T[q] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nx * ny; q += blockDim.x) {  // W(p, m), mode-major
    const int p = q % nx, m = q / nx;
    double s = 0.0;
    for (int j = 0; j < ny; ++j) s += by[m * ny + j] * T[p + nx * j];
    work[(int64_t)q * F.nz + r] = s;
  }
}

// One CTA per z-row of a member: phi = Bx^T W By of the row's modes.
template <class Out>
__global__ void __launch_bounds__(256) k_dir_inverse(DirectFac F, Out outb) {
  extern __shared__ double dsm[];
  const int b = blockIdx.x / F.nz;
  if (F.act && !F.act[b]) return;  // the whole CTA
  const Out out = outb.member(b);
  const double* work = F.work + (int64_t)b * F.nm * F.nz;
  const int nx = F.nx, ny = F.ny, r = blockIdx.x - b * F.nz;
  double* bx = dsm;
  double* by = bx + nx * nx;
  double* W = by + ny * ny;
  double* T = W + nx * ny;
  for (int q = threadIdx.x; q < nx * nx; q += blockDim.x) bx[q] = F.Bx[q];
  for (int q = threadIdx.x; q < ny * ny; q += blockDim.x) by[q] = F.By[q];
  for (int q = threadIdx.x; q < nx * ny; q += blockDim.x) W[q] = work[(int64_t)q * F.nz + r];
  __syncthreads();
  for (int q = threadIdx.x; q < nx * ny; q += blockDim.x) {  // T(i, m)
    const int i = q % nx, m = q / nx;
    double s = 0.0;
    for (int p = 0; p < nx; ++p) s += bx[p * nx + i] * W[p + nx * m];
    T[q] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nx * ny; q += blockDim.x) {  // phi(i, j)
    const int i = q % nx, j = q / nx;
    double s = 0.0;
    for (int m = 0; m < ny; ++m) s += by[m * ny + j] * T[i + nx * m];
    out.put(i, j, r, s);
  }
}

inline size_t dir_smem_bytes(int nx, int ny) {
  return (size_t)(nx * nx + ny * ny + 2 * nx * ny) * sizeof(double);
}

}  // namespace anel
