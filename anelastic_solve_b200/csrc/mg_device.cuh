// mg_device.cuh -- device code of the multigrid V-cycle, templated on the
// storage/arithmetic type T (double for the FP64 path, float for the FP32
// inner cycle of the mixed-precision solver).
//
// Layout: every level array is ghosted and column-major like the reference
// (i fastest); cell (i,j,k), 1-based with ghosts, sits at
// (i-1) + X*((j-1) + Y*(k-1)).  The FP64 instantiation is compiled with
// -fmad=false and evaluates every sum in the reference's left-to-right
// order, so its results are bit-identical to the Fortran semantics.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "anel_internal.h"

namespace anel {

template <typename T>
struct DevLevel {
  int nx, ny, nz;  // interior cells
  int X, Y, Z;     // ghosted dims
  int64_t XY, G;
  T* phi;
  T* src;
  const T* coef;   // cx1[X] cx2[X] cy3[Y] cy4[Y] cz5[Z] cz6[Z] dz5[Z] dz6[Z]
  BdryRule rule;
  // optional ghost table of a homogeneous rule (all boundary values 0):
  // gtab[g] = {ghost cell, interior cell it copies or -1 for 0}; null = the
  // rule is evaluated by ghost_value
  const int2* gtab;
};

template <typename T>
__device__ __forceinline__ const T* cx1p(const DevLevel<T>& L) { return L.coef; }
template <typename T>
__device__ __forceinline__ const T* cx2p(const DevLevel<T>& L) { return L.coef + L.X; }
template <typename T>
__device__ __forceinline__ const T* cy3p(const DevLevel<T>& L) { return L.coef + 2 * L.X; }
template <typename T>
__device__ __forceinline__ const T* cy4p(const DevLevel<T>& L) { return L.coef + 2 * L.X + L.Y; }
template <typename T>
__device__ __forceinline__ const T* cz5p(const DevLevel<T>& L) { return L.coef + 2 * L.X + 2 * L.Y; }
template <typename T>
__device__ __forceinline__ const T* cz6p(const DevLevel<T>& L) {
  return L.coef + 2 * L.X + 2 * L.Y + L.Z;
}
template <typename T>
__device__ __forceinline__ const T* dz5p(const DevLevel<T>& L) {
  return L.coef + 2 * L.X + 2 * L.Y + 2 * L.Z;
}
template <typename T>
__device__ __forceinline__ const T* dz6p(const DevLevel<T>& L) {
  return L.coef + 2 * L.X + 2 * L.Y + 3 * L.Z;
}

__device__ __forceinline__ int64_t cidx(int i, int j, int k, int X, int64_t XY) {
  return (int64_t)(i - 1) + (int64_t)X * (j - 1) + XY * (k - 1);
}

// ------------------------------------------------------------ ghost rule
// Final value of ghost cell (i,j,k) after the reference's serial mg_bdry
// (mg_bdry.F90:72-190): full periodic wrap X1, X2, X3, then the wall faces
// X2max, X3min, X2min, X3max, X1min, X1max, each over its full plane.  The
// value is found by walking the phases backwards to the interior cell it
// derives from, then replaying the Neumann additions forwards.  Reads only
// interior cells, so it can run concurrently with other ghost writers.
template <typename T>
__device__ __forceinline__ T ghost_value(const DevLevel<T>& L, const T* __restrict__ phi, int i, int j,
                                         int k) {
  const BdryRule& R = L.rule;
  T add[9];
  int sgn[9];
  int nops = 0;
  int t = 9;
  const int X = L.X, Y = L.Y, Z = L.Z;
  T base = T(0);
  for (;;) {
    int p = 0;
    if (t >= 9 && R.type[5] && i == X) p = 9;
    else if (t >= 8 && R.type[4] && i == 1) p = 8;
    else if (t >= 7 && R.type[3] && k == Z) p = 7;
    else if (t >= 6 && R.type[2] && j == 1) p = 6;
    else if (t >= 5 && R.type[1] && k == 1) p = 5;
    else if (t >= 4 && R.type[0] && j == Y) p = 4;
    else if (t >= 3 && (k == 1 || k == Z)) p = 3;
    else if (t >= 2 && (j == 1 || j == Y)) p = 2;
    else if (t >= 1 && (i == 1 || i == X)) p = 1;
    if (p == 0) {
      base = phi[cidx(i, j, k, X, L.XY)];
      break;
    }
    if (p >= 4) {
      const int face = p - 4;  // 0..5 in mg_bdry order
      if (R.type[face] == 2) {
        base = (T)R.val[face];
        break;
      }
      // Neumann: ghost = neighbour +/- phibc*d (X2max, X3max, X1max add)
      const T prod = (T)R.val[face] * (T)R.dist[face];
      add[nops] = prod;
      sgn[nops] = (face == 0 || face == 3 || face == 5) ? 1 : -1;
      ++nops;
      switch (face) {
        case 0: j = Y - 1; break;
        case 1: k = 2; break;
        case 2: j = 2; break;
        case 3: k = Z - 1; break;
        case 4: i = 2; break;
        default: i = X - 1; break;
      }
    } else if (p == 3) {
      k = (k == 1) ? Z - 1 : 2;
    } else if (p == 2) {
      j = (j == 1) ? Y - 1 : 2;
    } else {
      i = (i == 1) ? X - 1 : 2;
    }
    t = p - 1;
  }
  T v = base;
  for (int q = nops - 1; q >= 0; --q) v = (sgn[q] > 0) ? (v + add[q]) : (v - add[q]);
  return v;
}

// Map a linear ghost id (0 .. G-N-1) to a ghost cell: k-ghost planes, then
// j-ghost rows of interior k, then i-ghost columns of interior j,k.
__device__ __forceinline__ void ghost_cell(int64_t g, int X, int Y, int Z, int& i, int& j, int& k) {
  const int64_t XY = (int64_t)X * Y;
  if (g < 2 * XY) {
    const int64_t r = g % XY;
    k = (g < XY) ? 1 : Z;
    i = 1 + (int)(r % X);
    j = 1 + (int)(r / X);
    return;
  }
  g -= 2 * XY;
  const int nz = Z - 2;
  const int64_t Xnz = (int64_t)X * nz;
  if (g < 2 * Xnz) {
    const int64_t r = g % Xnz;
    j = (g < Xnz) ? 1 : Y;
    i = 1 + (int)(r % X);
    k = 2 + (int)(r / X);
    return;
  }
  g -= 2 * Xnz;
  const int ny = Y - 2;
  const int64_t nynz = (int64_t)ny * nz;
  const int64_t r = g % nynz;
  i = (g < nynz) ? 1 : X;
  j = 2 + (int)(r % ny);
  k = 2 + (int)(r / ny);
}

// Source of ghost cell (i,j,k) under a homogeneous rule: the walk of
// ghost_value without its arithmetic.  With every boundary value 0 the
// Neumann additions vanish, so the ghost is a copy of the interior cell the
// walk ends on, or 0 when it ends on a Dirichlet face.
template <typename T>
__device__ __forceinline__ int64_t ghost_source(const DevLevel<T>& L, int i, int j, int k) {
  const BdryRule& R = L.rule;
  int t = 9;
  const int X = L.X, Y = L.Y, Z = L.Z;
  for (;;) {
    int p = 0;
    if (t >= 9 && R.type[5] && i == X) p = 9;
    else if (t >= 8 && R.type[4] && i == 1) p = 8;
    else if (t >= 7 && R.type[3] && k == Z) p = 7;
    else if (t >= 6 && R.type[2] && j == 1) p = 6;
    else if (t >= 5 && R.type[1] && k == 1) p = 5;
    else if (t >= 4 && R.type[0] && j == Y) p = 4;
    else if (t >= 3 && (k == 1 || k == Z)) p = 3;
    else if (t >= 2 && (j == 1 || j == Y)) p = 2;
    else if (t >= 1 && (i == 1 || i == X)) p = 1;
    if (p == 0) return cidx(i, j, k, X, L.XY);
    if (p >= 4) {
      const int face = p - 4;
      if (R.type[face] == 2) return -1;
      switch (face) {
        case 0: j = Y - 1; break;
        case 1: k = 2; break;
        case 2: j = 2; break;
        case 3: k = Z - 1; break;
        case 4: i = 2; break;
        default: i = X - 1; break;
      }
    } else if (p == 3) {
      k = (k == 1) ? Z - 1 : 2;
    } else if (p == 2) {
      j = (j == 1) ? Y - 1 : 2;
    } else {
      i = (i == 1) ? X - 1 : 2;
    }
    t = p - 1;
  }
}

// Fill the ghost table of a level with a homogeneous rule (G < 2^31).
template <typename T>
__global__ void k_ghost_table(DevLevel<T> L, int2* __restrict__ tab) {
  const int64_t nghost = L.G - (int64_t)L.nx * L.ny * L.nz;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < nghost;
       g += (int64_t)gridDim.x * blockDim.x) {
    int i, j, k;
    ghost_cell(g, L.X, L.Y, L.Z, i, j, k);
    tab[g] = make_int2((int)cidx(i, j, k, L.X, L.XY), (int)ghost_source(L, i, j, k));
  }
}

// Ghost cells t0, t0+stride, ... of level L (the body of k_bdry).
template <typename T>
__device__ __forceinline__ void bdry_range(const DevLevel<T>& L, T* __restrict__ phi, int64_t t0,
                                           int64_t stride) {
  const int64_t nghost = L.G - (int64_t)L.nx * L.ny * L.nz;
  if (L.gtab) {
    for (int64_t g = t0; g < nghost; g += stride) {
      const int2 e = L.gtab[g];
      phi[e.x] = e.y >= 0 ? phi[e.y] : T(0);
    }
    return;
  }
  for (int64_t g = t0; g < nghost; g += stride) {
    int i, j, k;
    ghost_cell(g, L.X, L.Y, L.Z, i, j, k);
    phi[cidx(i, j, k, L.X, L.XY)] = ghost_value(L, phi, i, j, k);
  }
}

template <typename T>
__global__ void k_bdry(DevLevel<T> L, T* __restrict__ phi) {
  bdry_range(L, phi, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
}

// ------------------------------------------------------------- RB sweep
// One half-sweep of mg_relaxRB (mg_relax.F90:146-168): updates the cells
// with (i+j+k) % 2 == color (pass 1 = colour 0).  Reads only the other
// colour and ghosts, so the cells of one colour are independent.
template <typename T>
__device__ __forceinline__ T stencil_update(const DevLevel<T>& L, const T* __restrict__ phi, T s,
                                            int64_t c, int i, int j, int k) {
  const T a1 = cx1p(L)[i - 1], a2 = cx2p(L)[i - 1];
  const T a3 = cy3p(L)[j - 1], a4 = cy4p(L)[j - 1];
  const T a5 = cz5p(L)[k - 1], a6 = cz6p(L)[k - 1];
  const T diag = -(a1 + a2 + a3 + a4 + dz5p(L)[k - 1] + dz6p(L)[k - 1]);
  T acc = a1 * phi[c - 1];
  acc = acc + a2 * phi[c + 1];
  acc = acc + a3 * phi[c - L.X];
  acc = acc + a4 * phi[c + L.X];
  acc = acc + a5 * phi[c - L.XY];
  acc = acc + a6 * phi[c + L.XY];
  return (s - acc) / diag;
}

template <typename T>
__global__ void k_rb_sweep(DevLevel<T> L, int color) {
  const int hx = (L.nx + 1) >> 1;
  const int64_t total = (int64_t)hx * L.ny * L.nz;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int q = (int)(t % hx);
    const int64_t r = t / hx;
    const int j = 2 + (int)(r % L.ny);
    const int k = 2 + (int)(r / L.ny);
    const int i = 2 + ((color + j + k) & 1) + 2 * q;
    if (i > L.nx + 1) continue;
    const int64_t c = cidx(i, j, k, L.X, L.XY);
    L.phi[c] = stencil_update(L, L.phi, L.src[c], c, i, j, k);
  }
}

// -------------------------------------------------------- z-line sweep
// ZLINE smoother: one (i+j) colour of red-black z-line Gauss-Seidel
// (colour 0 = (i+j) even, the reference's first pass of mg_relaxLz,
// mg_relax.F90:487-535) with the level's own 7-point operator.  Each line
// is the tridiagonal (a = c5, b = c7, c = c6) solved by the Thomas routine
// of mg_relax.F90:541-595; for x/y-uniform coefficients its elimination is
// the same on every column, so only the substitution runs here:
//   G(1) = r(1), G(k) = r(k) + ap(k) G(k-1), phi(n) = G(n)/bp(n),
//   phi(k) = (G(k) - c(k) phi(k+1)) / bp(k).
// G is kept in the line's own cells (no other thread reads them in this
// colour).  One thread per pair of adjacent columns (i0, i0+1), which holds
// one column of each colour.
template <typename T>
struct ZFac {
  const T* ap;  // eliminated sub-diagonal, per k (index k-1; k = 2..nz+1 used)
  const T* bp;  // eliminated diagonal
};

// kLJ: the reference's mg_relaxLz boundary rows (mg_relax.F90:514-520):
// the ghost term sits inside the neighbour sum, and with one row only the
// top row's form is kept.
template <typename T, bool kLJ>
__global__ void k_zline(DevLevel<T> L, int color, ZFac<T> F) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;  // pair index
  const int j = 2 + blockIdx.y;
  const int i0 = 2 + 2 * p;
  if (i0 > L.nx + 1) return;
  const int i = i0 + ((color + i0 + j) & 1);
  if (i > L.nx + 1) return;
  const T a1 = cx1p(L)[i - 1], a2 = cx2p(L)[i - 1];
  const T a3 = cy3p(L)[j - 1], a4 = cy4p(L)[j - 1];
  const T* __restrict__ cz5 = cz5p(L);
  const T* __restrict__ cz6 = cz6p(L);
  T* phi = L.phi;
  const T* __restrict__ src = L.src;
  const int nz = L.nz;
  const int64_t X = L.X, XY = L.XY;
  const int64_t c0 = cidx(i, j, 1, L.X, L.XY);
  // forward substitution, k = 2 .. nz+1, in blocks of U rows whose loads
  // are all issued before the dependent recurrence (software pipelining)
  constexpr int U = 8;
  T g = T(0);
  for (int kb = 2; kb <= nz + 1; kb += U) {
    T r[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kb + u;
      if (k <= nz + 1) {
        const int64_t c = c0 + (int64_t)(k - 1) * XY;
        if (kLJ) {
          T sum = a1 * phi[c - 1] + a2 * phi[c + 1] + a3 * phi[c - X] + a4 * phi[c + X];
          if (k == nz + 1) sum = sum + cz6[nz] * phi[c + XY];
          else if (k == 2) sum = sum + cz5[1] * phi[c - XY];
          r[u] = src[c] - sum;
        } else {
          r[u] = src[c] - (a1 * phi[c - 1] + a2 * phi[c + 1] + a3 * phi[c - X] + a4 * phi[c + X]);
          if (k == 2) r[u] = r[u] - cz5[1] * phi[c - XY];
          if (k == nz + 1) r[u] = r[u] - cz6[nz] * phi[c + XY];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kb + u;
      if (k <= nz + 1) {
        g = (k == 2) ? r[u] : r[u] + F.ap[k - 1] * g;
        phi[c0 + (int64_t)(k - 1) * XY] = g;
      }
    }
  }
  // back substitution in blocks of U rows (loads of G first)
  T x = g / F.bp[nz];
  phi[c0 + (int64_t)nz * XY] = x;
  for (int kb = nz; kb >= 2; kb -= U) {
    T gv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kb - u;
      if (k >= 2) gv[u] = phi[c0 + (int64_t)(k - 1) * XY];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kb - u;
      if (k >= 2) {
        x = (gv[u] - cz6[k - 1] * x) / F.bp[k - 1];
        phi[c0 + (int64_t)(k - 1) * XY] = x;
      }
    }
  }
}

// Warp-per-line z-line smoother for levels with few columns (FP32 path):
// the line's tridiagonal system is solved by parallel cyclic reduction in
// shared memory (log2(nz) steps, each row updated from its neighbours at
// distance 2^s), so the latency is that of a few loads instead of a
// 2*nz-long dependent chain.  Not bit-matched to the Thomas order; used
// only inside the FP32 V-cycle of the mixed-precision solver.
template <typename T, int NMAX>
__global__ void k_zline_pcr(DevLevel<T> L, int color) {
  extern __shared__ unsigned char zl_smem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int nz = L.nz;
  T* sm = reinterpret_cast<T*>(zl_smem) + (size_t)wib * 4 * NMAX;
  T* A = sm;
  T* B = sm + NMAX;
  T* C = sm + 2 * NMAX;
  T* D = sm + 3 * NMAX;
  const int pairs = (L.nx + 1) >> 1;
  const int t = blockIdx.x * (blockDim.x >> 5) + wib;  // column of this colour
  if (t >= pairs * L.ny) return;
  const int j = 2 + t / pairs;
  const int i0 = 2 + 2 * (t % pairs);
  const int i = i0 + ((color + i0 + j) & 1);
  if (i > L.nx + 1) return;
  const T a1 = cx1p(L)[i - 1], a2 = cx2p(L)[i - 1];
  const T a3 = cy3p(L)[j - 1], a4 = cy4p(L)[j - 1];
  const T* cz5 = cz5p(L);
  const T* cz6 = cz6p(L);
  const T* d5 = dz5p(L);
  const T* d6 = dz6p(L);
  const int64_t X = L.X, XY = L.XY;
  const int64_t c0 = cidx(i, j, 1, L.X, L.XY);
  const T* phi = L.phi;
  for (int q = lane; q < nz; q += 32) {
    const int k = q + 2;
    const int64_t c = c0 + (int64_t)(k - 1) * XY;
    T d = L.src[c] - (a1 * phi[c - 1] + a2 * phi[c + 1] + a3 * phi[c - X] + a4 * phi[c + X]);
    T a = cz5[k - 1], cc = cz6[k - 1];
    if (q == 0) {
      d -= a * phi[c - XY];
      a = T(0);
    }
    if (q == nz - 1) {
      d -= cc * phi[c + XY];
      cc = T(0);
    }
    A[q] = a;
    C[q] = cc;
    B[q] = -(a1 + a2 + a3 + a4 + d5[k - 1] + d6[k - 1]);
    D[q] = d;
  }
  __syncwarp();
  constexpr int R = NMAX / 32;
  for (int st = 1; st < nz; st <<= 1) {
    T na[R], nb[R], nc[R], nd[R];
#pragma unroll
    for (int u = 0; u < R; ++u) {
      const int q = lane + 32 * u;
      if (q < nz) {
        T a = A[q], b = B[q], cc = C[q], d = D[q];
        if (q - st >= 0) {
          const T al = -a / B[q - st];
          b += al * C[q - st];
          d += al * D[q - st];
          a = al * A[q - st];
        } else {
          a = T(0);
        }
        if (q + st < nz) {
          const T be = -cc / B[q + st];
          b += be * A[q + st];
          d += be * D[q + st];
          cc = be * C[q + st];
        } else {
          cc = T(0);
        }
        na[u] = a;
        nb[u] = b;
        nc[u] = cc;
        nd[u] = d;
      }
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < R; ++u) {
      const int q = lane + 32 * u;
      if (q < nz) {
        A[q] = na[u];
        B[q] = nb[u];
        C[q] = nc[u];
        D[q] = nd[u];
      }
    }
    __syncwarp();
  }
  for (int q = lane; q < nz; q += 32) L.phi[c0 + (int64_t)(q + 1) * XY] = D[q] / B[q];
}

// Partitioned z-line smoother for the FP32 cycle.  Every line of a level
// has the same tridiagonal matrix (x/y-uniform coefficients), so the line
// is cut into P segments of m <= MR rows whose factors are precomputed on
// the host:
//   phase 1  each segment solves its own rows with the eliminated factors
//            (ap, 1/bp) ignoring its neighbours -> y, held in registers;
//   phase 2  the 2P interface values (first and last row of every segment)
//            follow from y by the precomputed inverse of the interface
//            system, z = Minv * yb;
//   phase 3  x = y + u * L(s-1) + v * F(s+1) with the precomputed influence
//            vectors u (response to the row before the segment) and v,
//            written once.
// A CTA holds 32 lines (lanes) x P segments (warps); each row is read
// (source and the four horizontal neighbours) and written exactly once and
// the dependent chain is 2m rows instead of 2n.  Not bit-matched to the
// Thomas order (the FP64 path keeps that).
template <typename T>
struct SegFac {
  const T* ap;    // segment-local eliminated sub-diagonal, per row (index k-1)
  const T* rbp;   // reciprocal of the segment-local eliminated diagonal
  const T* u;     // influence of the row before the segment
  const T* v;     // influence of the row after the segment
  const T* minv;  // (2P x 2P) inverse of the interface system, row major
  // ghost copies written by the sweep itself (homogeneous rule), or null:
  // img[3*((i-2) + nx*(j-2)) + e] = offset of the e-th ghost column that
  // copies line (i,j) (kNoImage: none); z1/zZ = source of the k=1 / k=Z
  // ghost of every column (0: zero, 1: row k=2, 2: row k=nz+1)
  const int* img;
  int z1, zZ;
  // cyclic-reduction multipliers of the level's line matrix (k_zline_cr),
  // or null: crs steps of alpha[nz] and gamma[nz], then 1/b[nz]
  const T* cr;
  int crs;
};
constexpr int kNoImage = -2147483647 - 1;

// Shared state of the partitioned solver: the line factors of the level,
// staged once per CTA (uniform across the lanes: shared-memory broadcasts
// instead of dependent global loads) and the interface values.
template <typename T, int P, int MR>
struct ZSegShared {
  T ap[P * MR], rbp[P * MR], c6[P * MR], u[P * MR], v[P * MR];
  T yb[32][2 * P + 1];
};

template <typename T, int P, int MR>
__device__ __forceinline__ void zseg_stage(const DevLevel<T>& L, const SegFac<T>& F,
                                           ZSegShared<T, P, MR>& S) {
  const T* __restrict__ cz6 = cz6p(L);
  for (int q = threadIdx.y * 32 + threadIdx.x; q < L.nz; q += 32 * P) {
    S.ap[q] = F.ap[q + 1];
    S.rbp[q] = F.rbp[q + 1];
    S.c6[q] = cz6[q + 1];
    S.u[q] = F.u[q + 1];
    S.v[q] = F.v[q + 1];
  }
}

// Lines t0 .. t0+31 of one colour (lane = line, threadIdx.y = segment),
// after zseg_stage by every thread of the CTA; ys holds MR * P * 32
// elements laid out [row][segment][lane] (each warp touches 32 consecutive
// words: no bank conflicts).  Contains two __syncthreads, so the whole CTA
// calls it together; the first one also publishes the staged factors and
// ends every thread's use of S from a previous call.
template <typename T, int P, int MR>
__device__ __forceinline__ void zseg_chunk(const DevLevel<T>& L, int color, const SegFac<T>& F,
                                           ZSegShared<T, P, MR>& S, T* ys, int64_t t0) {
  const int lane = threadIdx.x;  // line within the chunk
  const int s = threadIdx.y;     // segment
  const int n = L.nz;
  const int pairs = (L.nx + 1) >> 1;
  const int64_t t = t0 + lane;
  bool active = t < (int64_t)pairs * L.ny;
  int i = 0, j = 0;
  if (active) {
    j = 2 + (int)(t / pairs);
    const int i0 = 2 + 2 * (int)(t % pairs);
    i = i0 + ((color + i0 + j) & 1);
    active = i <= L.nx + 1;
  }
  const int m = n / P;
  const int lo = s * m;  // rows [lo, lo+m) of the line (row q <-> k = q+2)
  const int64_t X = L.X, XY = L.XY;
  const int64_t c0 = active ? cidx(i, j, 2, L.X, L.XY) + (int64_t)lo * XY : 0;
  T* yrow = ys + s * 32 + lane;  // row w at yrow[w * P * 32]
  constexpr int YS = P * 32;
  // residual rows of the segment (loads only; the factors are not needed)
  if (active) {
    const T a1 = cx1p(L)[i - 1], a2 = cx2p(L)[i - 1];
    const T a3 = cy3p(L)[j - 1], a4 = cy4p(L)[j - 1];
    const T* __restrict__ phi = L.phi + c0;
    const T* __restrict__ src = L.src + c0;
#pragma unroll 8
    for (int w = 0; w < m; ++w) {
      const int c = w * (int)XY;  // < 2^31: m * XY is checked by the host
      yrow[w * YS] = src[c] - (a1 * phi[c - 1] + a2 * phi[c + 1] + a3 * phi[c - X] + a4 * phi[c + X]);
    }
    if (lo == 0) yrow[0] -= cz5p(L)[1] * phi[-XY];
    if (lo + m == n) yrow[(m - 1) * YS] -= cz6p(L)[n] * phi[(int64_t)(m - 1) * XY + XY];
  }
  __syncthreads();
  T yfirst = T(0), ylast = T(0);
  if (active) {
    T g = yrow[0];
    for (int w = 1; w < m; ++w) {
      g = yrow[w * YS] + S.ap[lo + w] * g;
      yrow[w * YS] = g;
    }
    T x = g * S.rbp[lo + m - 1];
    yrow[(m - 1) * YS] = x;
    ylast = x;
    for (int w = m - 2; w >= 0; --w) {
      x = (yrow[w * YS] - S.c6[lo + w] * x) * S.rbp[lo + w];
      yrow[w * YS] = x;
    }
    yfirst = x;
  }
  S.yb[lane][2 * s] = yfirst;
  S.yb[lane][2 * s + 1] = ylast;
  __syncthreads();
  if (active) {
    // the two interface values this segment needs: L(s-1) = z[2s-1] and
    // F(s+1) = z[2s+2], z = Minv * yb
    T Lprev = T(0), Fnext = T(0);
    if (s > 0) {
      const T* mr = F.minv + (size_t)(2 * s - 1) * (2 * P);
#pragma unroll
      for (int p = 0; p < 2 * P; ++p) Lprev += mr[p] * S.yb[lane][p];
    }
    if (s < P - 1) {
      const T* mr = F.minv + (size_t)(2 * s + 2) * (2 * P);
#pragma unroll
      for (int p = 0; p < 2 * P; ++p) Fnext += mr[p] * S.yb[lane][p];
    }
    T* phi = L.phi;
    if (!F.img) {
#pragma unroll 8
      for (int w = 0; w < m; ++w)
        phi[c0 + (int64_t)w * XY] = yrow[w * YS] + S.u[lo + w] * Lprev + S.v[lo + w] * Fnext;
    } else {
      const int* im = F.img + 3 * ((i - 2) + (int64_t)L.nx * (j - 2));
      const int d0 = im[0], d1 = im[1], d2 = im[2];
      T xfirst = T(0), xlast = T(0);
#pragma unroll 4
      for (int w = 0; w < m; ++w) {
        const T x = yrow[w * YS] + S.u[lo + w] * Lprev + S.v[lo + w] * Fnext;
        const int64_t c = c0 + (int64_t)w * XY;
        phi[c] = x;
        if (d0 != kNoImage) phi[c + d0] = x;
        if (d1 != kNoImage) phi[c + d1] = x;
        if (d2 != kNoImage) phi[c + d2] = x;
        if (w == 0) xfirst = x;
        if (w == m - 1) xlast = x;
      }
      // z ghosts of the column and of its images (rows k=1 and k=Z)
      auto zrow = [&](int code, bool own_first) -> T {
        if (code == 0) return T(0);
        if ((code == 1) == own_first) return own_first ? xfirst : xlast;
        // the other end of the line: interface value z[0] or z[2P-1]
        const T* mr = F.minv + (size_t)(code == 1 ? 0 : 2 * P - 1) * (2 * P);
        T acc = T(0);
        for (int p = 0; p < 2 * P; ++p) acc += mr[p] * S.yb[lane][p];
        return acc;
      };
      if (lo == 0) {
        const T g = zrow(F.z1, true);
        const int64_t c = c0 - XY;
        phi[c] = g;
        if (d0 != kNoImage) phi[c + d0] = g;
        if (d1 != kNoImage) phi[c + d1] = g;
        if (d2 != kNoImage) phi[c + d2] = g;
      }
      if (lo + m == n) {
        const T g = zrow(F.zZ, false);
        const int64_t c = c0 + (int64_t)m * XY;
        phi[c] = g;
        if (d0 != kNoImage) phi[c + d0] = g;
        if (d1 != kNoImage) phi[c + d1] = g;
        if (d2 != kNoImage) phi[c + d2] = g;
      }
    }
  }
}

template <typename T, int P, int MR>
__global__ void __launch_bounds__(32 * P, 2) k_zline_seg(DevLevel<T> L, int color, SegFac<T> F) {
  extern __shared__ unsigned char zs_smem[];
  __shared__ ZSegShared<T, P, MR> S;
  zseg_stage(L, F, S);
  zseg_chunk(L, color, F, S, reinterpret_cast<T*>(zs_smem), (int64_t)blockIdx.x * 32);
}

// ------------------------------------------ z-line solve, cyclic reduction
// Levels with few lines (the coarse levels of the FP32 cycle): one CTA per
// line, one thread per row.  Every line of a level has the same tridiagonal
// matrix, so the multipliers of parallel cyclic reduction are precomputed
// on the host: step s (stride 2^s) updates d_r += alpha_s[r] d_(r-2^s) +
// gamma_s[r] d_(r+2^s), and after the last step x_r = d_r / b_r.  The
// dependent chain is ceil(log2 nz) steps (the partitioned solver's is
// 2 x 32 rows), so a sweep over a handful of lines costs a few
// microseconds instead of one long per-thread chain.  The right-hand side
// and the ghost copies are those of k_zline_seg.
constexpr int kCRMaxSteps = 10;
constexpr int kCRMaxRows = 1 << kCRMaxSteps;
template <typename T>
__global__ void __launch_bounds__(kCRMaxRows) k_zline_cr(DevLevel<T> L, int color, SegFac<T> F) {
  __shared__ T D[2][kCRMaxRows];
  const int n = L.nz;
  const int pairs = (L.nx + 1) >> 1;
  const int t = blockIdx.x;  // line of this colour
  const int j = 2 + t / pairs;
  const int i0 = 2 + 2 * (t % pairs);
  const int i = i0 + ((color + i0 + j) & 1);
  if (i > L.nx + 1) return;  // the whole CTA: no barrier reached
  const int r = threadIdx.x;
  const bool row = r < n;
  const int64_t X = L.X, XY = L.XY;
  const int64_t cb = cidx(i, j, 2, L.X, L.XY);  // row 0 (k = 2)
  const int64_t c = cb + (int64_t)(row ? r : 0) * XY;
  T al[kCRMaxSteps], ga[kCRMaxSteps];
  T d = T(0), rb = T(0);
  if (row) {
    const T a1 = cx1p(L)[i - 1], a2 = cx2p(L)[i - 1];
    const T a3 = cy3p(L)[j - 1], a4 = cy4p(L)[j - 1];
    const T* __restrict__ phi = L.phi;
    d = L.src[c] - (a1 * phi[c - 1] + a2 * phi[c + 1] + a3 * phi[c - X] + a4 * phi[c + X]);
    if (r == 0) d -= cz5p(L)[1] * phi[c - XY];
    if (r == n - 1) d -= cz6p(L)[n] * phi[c + XY];
#pragma unroll
    for (int q = 0; q < kCRMaxSteps; ++q)
      if (q < F.crs) {
        al[q] = F.cr[(size_t)(2 * q) * n + r];
        ga[q] = F.cr[(size_t)(2 * q + 1) * n + r];
      }
    rb = F.cr[(size_t)(2 * F.crs) * n + r];
    D[0][r] = d;
  }
  __syncthreads();
  int b = 0;
#pragma unroll
  for (int q = 0; q < kCRMaxSteps; ++q) {
    if (q >= F.crs) break;  // uniform across the CTA
    const int st = 1 << q;
    if (row) {
      T v = d;
      if (r - st >= 0) v += al[q] * D[b][r - st];
      if (r + st < n) v += ga[q] * D[b][r + st];
      d = v;
      D[b ^ 1][r] = d;
    }
    b ^= 1;
    __syncthreads();  // (double buffer: one barrier per step)
  }
  const T x = d * rb;
  if (row) D[b ^ 1][r] = x;
  __syncthreads();
  if (!row) return;
  T* phi = L.phi;
  int d0 = kNoImage, d1 = kNoImage, d2 = kNoImage;
  if (F.img) {
    const int* im = F.img + 3 * ((i - 2) + (int64_t)L.nx * (j - 2));
    d0 = im[0];
    d1 = im[1];
    d2 = im[2];
  }
  auto put = [&](int64_t cc, T v) {
    phi[cc] = v;
    if (d0 != kNoImage) phi[cc + d0] = v;
    if (d1 != kNoImage) phi[cc + d1] = v;
    if (d2 != kNoImage) phi[cc + d2] = v;
  };
  put(c, x);
  if (F.img) {
    // z ghosts of the column and of its images (rows k=1 and k=Z)
    const T* xs = D[b ^ 1];
    auto zval = [&](int code) -> T { return code == 0 ? T(0) : (code == 1 ? xs[0] : xs[n - 1]); };
    if (r == 0) put(cb - XY, zval(F.z1));
    if (r == n - 1) put(cb + (int64_t)n * XY, zval(F.zZ));
  }
}

// ----------------------------------------------------- residual + restrict
// mg_restr.F90:114-241.  One thread per coarse cell (ghosts included):
// coarse phi <- 0 everywhere, coarse f <- 0 on ghosts and, on the interior,
// the scaled sum of the children's residuals res = f - A phi, summed in the
// reference order of the active variant.  cdir bit d set = direction d is
// coarsened between the two levels.
template <typename T>
__device__ __forceinline__ T fine_resid(const DevLevel<T>& F, int i, int j, int k) {
  const int64_t c = cidx(i, j, k, F.X, F.XY);
  const T a1 = cx1p(F)[i - 1], a2 = cx2p(F)[i - 1];
  const T a3 = cy3p(F)[j - 1], a4 = cy4p(F)[j - 1];
  const T a5 = cz5p(F)[k - 1], a6 = cz6p(F)[k - 1];
  const T diag = -(a1 + a2 + a3 + a4 + dz5p(F)[k - 1] + dz6p(F)[k - 1]);
  const T* __restrict__ p = F.phi;
  T acc = a1 * p[c - 1];
  acc = acc + a2 * p[c + 1];
  acc = acc + a3 * p[c - F.X];
  acc = acc + a4 * p[c + F.X];
  acc = acc + a5 * p[c - F.XY];
  acc = acc + a6 * p[c + F.XY];
  acc = acc + diag * p[c];
  return F.src[c] - acc;
}

// Value of interior coarse cell (ic,jc,kc) for the coarsening variant CD:
// the scaled sum of the children's residuals in the reference order.
template <typename T, int CD>
__device__ __forceinline__ T restrict_value(const DevLevel<T>& F, int ic, int jc, int kc) {
  constexpr bool cx = CD & 1, cy = CD & 2, cz = CD & 4;
  const int i = cx ? 2 * ic - 2 : ic;
  const int j = cy ? 2 * jc - 2 : jc;
  const int k = cz ? 2 * kc - 2 : kc;
  if constexpr (cx && cy && cz) {
    T s = fine_resid(F, i, j, k);
    s = s + fine_resid(F, i, j + 1, k);
    s = s + fine_resid(F, i, j, k + 1);
    s = s + fine_resid(F, i, j + 1, k + 1);
    s = s + fine_resid(F, i + 1, j, k);
    s = s + fine_resid(F, i + 1, j + 1, k + 1);
    s = s + fine_resid(F, i + 1, j + 1, k);
    s = s + fine_resid(F, i + 1, j, k + 1);
    return T(0.125) * s;
  } else if constexpr (!cx && !cy) {  // z only
    return T(0.5) * (fine_resid(F, i, j, k) + fine_resid(F, i, j, k + 1));
  } else if constexpr (!cx && !cz) {  // y only
    return T(0.5) * (fine_resid(F, i, j, k) + fine_resid(F, i, j + 1, k));
  } else if constexpr (!cy && !cz) {  // x only
    return T(0.5) * (fine_resid(F, i, j, k) + fine_resid(F, i + 1, j, k));
  } else if constexpr (!cx) {  // y,z
    T s = fine_resid(F, i, j, k);
    s = s + fine_resid(F, i, j + 1, k);
    s = s + fine_resid(F, i, j, k + 1);
    s = s + fine_resid(F, i, j + 1, k + 1);
    return T(0.25) * s;
  } else if constexpr (!cy) {  // x,z
    T s = fine_resid(F, i, j, k);
    s = s + fine_resid(F, i, j, k + 1);
    s = s + fine_resid(F, i + 1, j, k);
    s = s + fine_resid(F, i + 1, j, k + 1);
    return T(0.25) * s;
  } else {  // x,y
    T s = fine_resid(F, i, j, k);
    s = s + fine_resid(F, i + 1, j, k);
    s = s + fine_resid(F, i, j + 1, k);
    s = s + fine_resid(F, i + 1, j + 1, k);
    return T(0.25) * s;
  }
}

// kZBatch consecutive z-cells per thread, every load issued before the
// first store (a store to one array may not be moved past a load of
// another by the compiler, so interleaving would serialise the cells).
constexpr int kZBatch = 4;

// Coarse cells: grid (ceil(nx/128), Y, ceil(Z/kZBatch)); thread ic covers
// interior column ic, and the threads of columns 2 and nx+1 also zero the
// ghost columns 1 and nx+2.  Coarse phi <- 0 everywhere, coarse f <- 0 on
// ghosts.
template <typename T, int CD>
__global__ void __launch_bounds__(128) k_restrict(DevLevel<T> F, DevLevel<T> Cl) {
  const int ic = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  if (ic > Cl.nx + 1) return;
  const int jc = 1 + blockIdx.y;
  const int k0 = 1 + blockIdx.z * kZBatch;
  const bool row_in = jc >= 2 && jc <= Cl.ny + 1;
  T v[kZBatch];
  if (row_in && k0 >= 2 && k0 + kZBatch - 1 <= Cl.nz + 1) {
#pragma unroll
    for (int q = 0; q < kZBatch; ++q) v[q] = restrict_value<T, CD>(F, ic, jc, k0 + q);
  } else {
#pragma unroll
    for (int q = 0; q < kZBatch; ++q) {
      const int kc = k0 + q;
      v[q] = (row_in && kc >= 2 && kc <= Cl.nz + 1) ? restrict_value<T, CD>(F, ic, jc, kc) : T(0);
    }
  }
  const int64_t t0 = cidx(ic, jc, k0, Cl.X, Cl.XY);
  const bool g_lo = ic == 2, g_hi = ic == Cl.nx + 1;  // ghost columns beside this one
#pragma unroll
  for (int q = 0; q < kZBatch; ++q) {
    if (k0 + q > Cl.Z) break;
    const int64_t t = t0 + q * Cl.XY;
    Cl.phi[t] = T(0);
    Cl.src[t] = v[q];
    if (g_lo) {
      Cl.phi[t - 1] = T(0);
      Cl.src[t - 1] = T(0);
    }
    if (g_hi) {
      Cl.phi[t + 1] = T(0);
      Cl.src[t + 1] = T(0);
    }
  }
}

// -------------------------------------------------------------- prolong
// mg_cor.F90:102-290 for the fine interior (fine ghosts are rebuilt by the
// boundary pass that follows, as in the reference).  In a coarsened
// direction fine index f uses coarse ic = (f+1)/2 (f odd, near point ic) or
// ic = f/2 (f even, near point ic+1); weights 3 (near) and 1 (far).
template <typename T, int CD>
__device__ __forceinline__ T prolong_corr(const DevLevel<T>& Cl, int i, int j, int k) {
  constexpr bool cx = CD & 1, cy = CD & 2, cz = CD & 4;
  const int ic = cx ? ((i & 1) ? (i + 1) >> 1 : i >> 1) : i;
  const int jc = cy ? ((j & 1) ? (j + 1) >> 1 : j >> 1) : j;
  const int kc = cz ? ((k & 1) ? (k + 1) >> 1 : k >> 1) : k;
  // weight of coarse offset o (0/1) in each direction
  const T wx0 = cx ? ((i & 1) ? T(3) : T(1)) : T(1), wx1 = cx ? ((i & 1) ? T(1) : T(3)) : T(0);
  const T wy0 = cy ? ((j & 1) ? T(3) : T(1)) : T(1), wy1 = cy ? ((j & 1) ? T(1) : T(3)) : T(0);
  const T wz0 = cz ? ((k & 1) ? T(3) : T(1)) : T(1), wz1 = cz ? ((k & 1) ? T(1) : T(3)) : T(0);
  const T* __restrict__ pc = Cl.phi + cidx(ic, jc, kc, Cl.X, Cl.XY);
  const int64_t ox = 1, oy = Cl.X, oz = Cl.XY;
  if constexpr (cx && cy && cz) {
    // order (x,y,z) offsets: 000 010 001 011 100 110 101 111
    T s = (wx0 * wy0 * wz0) * pc[0];
    s = s + (wx0 * wy1 * wz0) * pc[oy];
    s = s + (wx0 * wy0 * wz1) * pc[oz];
    s = s + (wx0 * wy1 * wz1) * pc[oy + oz];
    s = s + (wx1 * wy0 * wz0) * pc[ox];
    s = s + (wx1 * wy1 * wz0) * pc[ox + oy];
    s = s + (wx1 * wy0 * wz1) * pc[ox + oz];
    s = s + (wx1 * wy1 * wz1) * pc[ox + oy + oz];
    return s / T(64);
  } else if constexpr (!cx && !cy) {  // z only
    return (wz0 * pc[0] + wz1 * pc[oz]) / T(4);
  } else if constexpr (!cx && !cz) {  // y only
    return (wy0 * pc[0] + wy1 * pc[oy]) / T(4);
  } else if constexpr (!cy && !cz) {  // x only
    return (wx0 * pc[0] + wx1 * pc[ox]) / T(4);
  } else if constexpr (!cx) {  // y,z: (y,z) 00 10 01 11
    T s = (wy0 * wz0) * pc[0];
    s = s + (wy1 * wz0) * pc[oy];
    s = s + (wy0 * wz1) * pc[oz];
    s = s + (wy1 * wz1) * pc[oy + oz];
    return s / T(16);
  } else if constexpr (!cy) {  // x,z: (x,z) 00 10 01 11
    T s = (wx0 * wz0) * pc[0];
    s = s + (wx1 * wz0) * pc[ox];
    s = s + (wx0 * wz1) * pc[oz];
    s = s + (wx1 * wz1) * pc[ox + oz];
    return s / T(16);
  } else {  // x,y: (x,y) 00 10 01 11
    T s = (wx0 * wy0) * pc[0];
    s = s + (wx1 * wy0) * pc[ox];
    s = s + (wx0 * wy1) * pc[oy];
    s = s + (wx1 * wy1) * pc[ox + oy];
    return s / T(16);
  }
}

// fine interior cells: grid (ceil(nx/128), ny, ceil(nz/kZBatch)); the
// corrections and old values of all kZBatch cells are loaded before the
// first store.
template <typename T, int CD>
__global__ void __launch_bounds__(128) k_prolong(DevLevel<T> F, DevLevel<T> Cl) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i > F.nx + 1) return;
  const int j = 2 + blockIdx.y;
  const int k0 = 2 + blockIdx.z * kZBatch;
  T* p = F.phi + cidx(i, j, k0, F.X, F.XY);
  const int64_t XY = F.XY;
  T val[kZBatch];
  if (k0 + kZBatch - 1 <= F.nz + 1) {
#pragma unroll
    for (int q = 0; q < kZBatch; ++q) val[q] = p[q * XY] + prolong_corr<T, CD>(Cl, i, j, k0 + q);
#pragma unroll
    for (int q = 0; q < kZBatch; ++q) p[q * XY] = val[q];
  } else {
#pragma unroll
    for (int q = 0; q < kZBatch; ++q)
      if (k0 + q <= F.nz + 1) val[q] = p[q * XY] + prolong_corr<T, CD>(Cl, i, j, k0 + q);
#pragma unroll
    for (int q = 0; q < kZBatch; ++q)
      if (k0 + q <= F.nz + 1) p[q * XY] = val[q];
  }
}

}  // namespace anel
