// mg_col.cuh -- the FP32 levels of the z-line cycle stored column by column.
//
// With the ZLINE smoother and x/y semi-coarsening every level keeps the fine
// grid's nz, every z-line is solved whole, and the transfers only combine
// columns.  So the FP32 levels of the mixed-precision cycle are stored with
// z fastest: column (i,j) (1-based ghosted) holds its nz+2 cells
// contiguously, padded to a stride of nz + 2*kColPad floats so that every
// column starts on a 32-byte sector and its interior rows on a sector too:
//   cell (i,j,k) at ((i-1) + X*(j-1)) * CS + (kColPad - 2) + k.
// A z-line is then 2 KB of consecutive memory (nz = 512): a warp reads it,
// and each of its four horizontal neighbours, with coalesced 128-byte
// accesses, and a colour's sweep moves the algorithmic 6 bytes per cell
// (the other colour's phi, this colour's f, this colour's new phi) with no
// half-used sectors.  The FP64 fine level keeps the reference layout; the
// defect-correction kernels (mg_col64.cu) transpose through shared memory.
//
// Line solve: one warp per line, lane s owning the M = nz/32 consecutive
// rows s*M .. s*M+M-1.  The last row of each lane is a separator; the M-1
// rows before it are solved by Thomas elimination with the two separators
// around them as unknowns (spikes L, R), which leaves a 32-unknown
// tridiagonal system in the separators, solved across the lanes by
// parallel cyclic reduction with shuffles.  The line matrix is the same for
// every line of a level (x/y-uniform coefficients, r = r(z)), so every
// factor and multiplier is precomputed on the host in FP64 and only the
// right-hand side flows through the kernel.
#pragma once

#include "mg_device.cuh"

namespace anel {

constexpr int kColPad = 8;
inline int col_stride(int nz) { return nz + 2 * kColPad; }

struct ColLevel {
  int nx, ny, nz;  // interior cells
  int X, Y;        // ghosted columns per direction
  int CS;          // column stride (floats)
  float* phi;
  float* src;
  float a1, a2, a3, a4;  // x/y line coefficients (uniform over the level)
  const float* cz5;      // z coefficients, indexed k-1 (Z values each)
  const float* cz6;
  const float* dz5;
  const float* dz6;
  // ghost copies written by the sweeps and the prolongation: three image
  // column offsets (in columns) per interior column, kNoImage for none;
  // z1 / zZ = source of the k = 1 / k = Z ghost of every column (0 zero,
  // 1 row k = 2, 2 row k = nz+1)
  const int* img;
  int z1, zZ;
};

__host__ __device__ __forceinline__ int64_t col_cell(const ColLevel& L, int i, int j, int k) {
  return ((int64_t)(i - 1) + (int64_t)L.X * (j - 1)) * L.CS + (kColPad - 2) + k;
}

// Floats of the per-level sweep factors for M rows per lane: five arrays
// [w][lane] over the M-1 inner rows (ap, 1/bp, sup, L, R), then [b][lane]
// for b = 0 sub(separator), 1 sup(separator), 2..6 PCR alpha_q, 7..11 PCR
// gamma_q, 12 1/b of the reduced separator system.
__host__ __device__ constexpr int col_fac_floats(int M) { return 5 * (M - 1) * 32 + 13 * 32; }

constexpr int kColWarps = 8;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int col_pad(int r) { return r + (r >> 5); }

// Writes v to row `c` of the column and of its image columns.
__device__ __forceinline__ void col_put(float* __restrict__ P, int64_t c, float v, int64_t o0, int64_t o1,
                                        int64_t o2, bool h0, bool h1, bool h2) {
  P[c] = v;
  if (h0) P[c + o0] = v;
  if (h1) P[c + o1] = v;
  if (h2) P[c + o2] = v;
}

// One colour of the z-line Gauss-Seidel sweep: lines (i,j) with
// (i + j) % 2 == color, in the pairing of k_zline_seg.  Each line's
// right-hand side takes the other colour's horizontal neighbours and the
// line's own z-ghosts as known; the new values are written with their
// ghost copies.
template <int M>
__global__ void __launch_bounds__(32 * kColWarps, 3) k_col_sweep(ColLevel L, int color,
                                                                 const float* __restrict__ fac) {
  constexpr int NF = col_fac_floats(M);
  constexpr int N = 32 * M;
  __shared__ float sf[NF];
  __shared__ float sy[kColWarps][N + M];
  for (int q = threadIdx.x; q < NF; q += blockDim.x) sf[q] = fac[q];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* ys = sy[warp];
  const float* Fap = sf;
  const float* Frbp = sf + (M - 1) * 32;
  const float* Fsup = sf + 2 * (M - 1) * 32;
  const float* FL = sf + 3 * (M - 1) * 32;
  const float* FR = sf + 4 * (M - 1) * 32;
  const float* Fg = sf + 5 * (M - 1) * 32;
  const float sub_h = Fg[lane], sup_h = Fg[32 + lane], rb = Fg[12 * 32 + lane];
  const int pairs = (L.nx + 1) >> 1;
  const int64_t nlines = (int64_t)pairs * L.ny;
  const int64_t CS = L.CS, XC = (int64_t)L.X * L.CS;
  const float a1 = L.a1, a2 = L.a2, a3 = L.a3, a4 = L.a4;
  const float c5b = L.cz5[1], c6t = L.cz6[L.nz];  // row 0 to its k=1 ghost, row n-1 to k=Z
  for (int64_t t = (int64_t)blockIdx.x * kColWarps + warp; t < nlines; t += (int64_t)gridDim.x * kColWarps) {
    const int j = 2 + (int)(t / pairs);
    const int i0 = 2 + 2 * (int)(t % pairs);
    const int i = i0 + ((color + i0 + j) & 1);
    if (i > L.nx + 1) continue;  // uniform across the warp
    const int64_t c0 = col_cell(L, i, j, 2);  // row 0
    const float* __restrict__ P = L.phi;
    const float* __restrict__ S = L.src;
    float v[M];
#pragma unroll
    for (int q = 0; q < M; ++q) {
      const int64_t c = c0 + lane + 32 * q;
      v[q] = S[c] - (a1 * P[c - CS] + a2 * P[c + CS] + a3 * P[c - XC] + a4 * P[c + XC]);
    }
    if (lane == 0) v[0] -= c5b * P[c0 - 1];
    if (lane == 31) v[M - 1] -= c6t * P[c0 + N];
    // row order -> segment order (lane s: rows s*M .. s*M+M-1)
#pragma unroll
    for (int q = 0; q < M; ++q) ys[col_pad(lane + 32 * q)] = v[q];
    __syncwarp();
    float y[M];
#pragma unroll
    for (int w = 0; w < M; ++w) y[w] = ys[col_pad(lane * M + w)];
    __syncwarp();
    // inner rows 0..M-2: local solution with both separators at zero
    float g = y[0];
#pragma unroll
    for (int w = 1; w < M - 1; ++w) {
      g = y[w] + Fap[w * 32 + lane] * g;
      y[w] = g;
    }
    float x = g * Frbp[(M - 2) * 32 + lane];
    y[M - 2] = x;
#pragma unroll
    for (int w = M - 3; w >= 0; --w) {
      x = (y[w] - Fsup[w * 32 + lane] * x) * Frbp[w * 32 + lane];
      y[w] = x;
    }
    // separator system across the lanes
    const float ynext = __shfl_down_sync(kFull, y[0], 1);
    float h = y[M - 1] - sub_h * y[M - 2] - (lane < 31 ? sup_h * ynext : 0.f);
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const int st = 1 << q;
      const float up = __shfl_up_sync(kFull, h, st);
      const float dn = __shfl_down_sync(kFull, h, st);
      h = h + Fg[(2 + q) * 32 + lane] * up + Fg[(7 + q) * 32 + lane] * dn;
    }
    const float xs = h * rb;
    const float xprev = __shfl_up_sync(kFull, xs, 1);  // lane 0: L = 0
#pragma unroll
    for (int w = 0; w < M - 1; ++w) y[w] = y[w] + FL[w * 32 + lane] * xprev + FR[w * 32 + lane] * xs;
    y[M - 1] = xs;
    // segment order -> row order
#pragma unroll
    for (int w = 0; w < M; ++w) ys[col_pad(lane * M + w)] = y[w];
    __syncwarp();
#pragma unroll
    for (int q = 0; q < M; ++q) v[q] = ys[col_pad(lane + 32 * q)];
    __syncwarp();
    int d0 = kNoImage, d1 = kNoImage, d2 = kNoImage;
    if (L.img) {
      const int* im = L.img + 3 * ((i - 2) + (int64_t)L.nx * (j - 2));
      d0 = im[0];
      d1 = im[1];
      d2 = im[2];
    }
    const bool h0 = d0 != kNoImage, h1 = d1 != kNoImage, h2 = d2 != kNoImage;
    const int64_t o0 = h0 ? (int64_t)d0 * CS : 0, o1 = h1 ? (int64_t)d1 * CS : 0,
                  o2 = h2 ? (int64_t)d2 * CS : 0;
    float* __restrict__ Pw = L.phi;
#pragma unroll
    for (int q = 0; q < M; ++q) col_put(Pw, c0 + lane + 32 * q, v[q], o0, o1, o2, h0, h1, h2);
    // z ghosts of the column and of its images
    const float r0 = __shfl_sync(kFull, v[0], 0);
    const float rn = __shfl_sync(kFull, v[M - 1], 31);
    if (lane == 0 || lane == 31) {
      const int code = lane == 0 ? L.z1 : L.zZ;
      const float gv = code == 0 ? 0.f : (code == 1 ? r0 : rn);
      col_put(Pw, lane == 0 ? c0 - 1 : c0 + N, gv, o0, o1, o2, h0, h1, h2);
    }
  }
}

// Residual f - A phi of fine cell (i,j,k), in the order of fine_resid.
__device__ __forceinline__ float col_resid(const ColLevel& F, int i, int j, int k) {
  const int64_t c = col_cell(F, i, j, k);
  const float* __restrict__ p = F.phi;
  const int64_t XC = (int64_t)F.X * F.CS;
  const float diag = -(F.a1 + F.a2 + F.a3 + F.a4 + F.dz5[k - 1] + F.dz6[k - 1]);
  float acc = F.a1 * p[c - F.CS];
  acc = acc + F.a2 * p[c + F.CS];
  acc = acc + F.a3 * p[c - XC];
  acc = acc + F.a4 * p[c + XC];
  acc = acc + F.cz5[k - 1] * p[c - 1];
  acc = acc + F.cz6[k - 1] * p[c + 1];
  acc = acc + diag * p[c];
  return F.src[c] - acc;
}

// mg_restr's x/y variants (z is not coarsened): coarse f of interior cell
// (ic,jc,k) from the residuals of its children, in restrict_value's order.
// Grid (coarse interior columns, ceil(nz/128)); the caller zeroes coarse phi.
template <int CD>
__global__ void __launch_bounds__(128) k_col_restrict(ColLevel F, ColLevel C) {
  const int k = 2 + blockIdx.y * 128 + threadIdx.x;
  if (k > C.nz + 1) return;
  const int64_t col = blockIdx.x;
  const int ic = 2 + (int)(col % C.nx), jc = 2 + (int)(col / C.nx);
  constexpr bool cx = CD & 1, cy = CD & 2;
  const int i = cx ? 2 * ic - 2 : ic;
  const int j = cy ? 2 * jc - 2 : jc;
  float v;
  if constexpr (cx && cy) {
    float s = col_resid(F, i, j, k);
    s = s + col_resid(F, i + 1, j, k);
    s = s + col_resid(F, i, j + 1, k);
    s = s + col_resid(F, i + 1, j + 1, k);
    v = 0.25f * s;
  } else if constexpr (cx) {
    v = 0.5f * (col_resid(F, i, j, k) + col_resid(F, i + 1, j, k));
  } else {
    v = 0.5f * (col_resid(F, i, j, k) + col_resid(F, i, j + 1, k));
  }
  C.src[col_cell(C, ic, jc, k)] = v;
}

// mg_cor's x/y variants for the fine interior, in prolong_corr's order,
// with the ghost copies of the updated cells written alongside (the
// boundary pass of the row-major cycle).  Grid (fine interior columns,
// ceil(nz/128)).
template <int CD>
__global__ void __launch_bounds__(128) k_col_prolong(ColLevel F, ColLevel C) {
  const int k = 2 + blockIdx.y * 128 + threadIdx.x;
  if (k > F.nz + 1) return;
  const int64_t col = blockIdx.x;
  const int i = 2 + (int)(col % F.nx), j = 2 + (int)(col / F.nx);
  constexpr bool cx = CD & 1, cy = CD & 2;
  const int ic = cx ? ((i + 1) >> 1) : i;
  const int jc = cy ? ((j + 1) >> 1) : j;
  const float wx0 = cx ? ((i & 1) ? 3.f : 1.f) : 1.f, wx1 = cx ? ((i & 1) ? 1.f : 3.f) : 0.f;
  const float wy0 = cy ? ((j & 1) ? 3.f : 1.f) : 1.f, wy1 = cy ? ((j & 1) ? 1.f : 3.f) : 0.f;
  const float* __restrict__ pc = C.phi + col_cell(C, ic, jc, k);
  const int64_t ox = C.CS, oy = (int64_t)C.X * C.CS;
  float corr;
  if constexpr (cx && cy) {
    float s = (wx0 * wy0) * pc[0];
    s = s + (wx1 * wy0) * pc[ox];
    s = s + (wx0 * wy1) * pc[oy];
    s = s + (wx1 * wy1) * pc[ox + oy];
    corr = s / 16.f;
  } else if constexpr (cx) {
    corr = (wx0 * pc[0] + wx1 * pc[ox]) / 4.f;
  } else {
    corr = (wy0 * pc[0] + wy1 * pc[oy]) / 4.f;
  }
  const int64_t c = col_cell(F, i, j, k);
  float* __restrict__ P = F.phi;
  const float v = P[c] + corr;
  int d0 = kNoImage, d1 = kNoImage, d2 = kNoImage;
  if (F.img) {
    const int* im = F.img + 3 * ((i - 2) + (int64_t)F.nx * (j - 2));
    d0 = im[0];
    d1 = im[1];
    d2 = im[2];
  }
  const bool h0 = d0 != kNoImage, h1 = d1 != kNoImage, h2 = d2 != kNoImage;
  const int64_t o0 = h0 ? (int64_t)d0 * F.CS : 0, o1 = h1 ? (int64_t)d1 * F.CS : 0,
                o2 = h2 ? (int64_t)d2 * F.CS : 0;
  col_put(P, c, v, o0, o1, o2, h0, h1, h2);
  // z ghosts: the k = 2 thread writes the ghosts that copy row k = 2 or
  // are zero, the k = nz+1 thread those that copy row k = nz+1
  const int64_t g1 = c - (k - 1), gZ = c + (F.nz + 2 - k);
  if (k == 2) {
    if (F.z1 != 2) col_put(P, g1, F.z1 == 1 ? v : 0.f, o0, o1, o2, h0, h1, h2);
    if (F.zZ != 2) col_put(P, gZ, F.zZ == 1 ? v : 0.f, o0, o1, o2, h0, h1, h2);
  }
  if (k == F.nz + 1) {
    if (F.z1 == 2) col_put(P, g1, v, o0, o1, o2, h0, h1, h2);
    if (F.zZ == 2) col_put(P, gZ, v, o0, o1, o2, h0, h1, h2);
  }
}

}  // namespace anel
