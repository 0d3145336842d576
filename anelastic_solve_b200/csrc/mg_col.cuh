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
  // members of a batch (independent problems on the same level): member m's
  // columns start at phi / src + m * ms; act[m] == 0 leaves member m alone
  // (null: every member is active)
  int nm = 1;
  int64_t ms = 0;
  const int* act = nullptr;
};

// FP64 fine arrays of one member of a batch (reference layout)
struct MemberIO {
  double* phi;
  const double* rhs;
};

// the level of member m alone (its arrays; nm = 1)
__host__ __device__ __forceinline__ ColLevel col_member(ColLevel L, int m) {
  L.phi += m * L.ms;
  L.src += m * L.ms;
  L.nm = 1;
  return L;
}
__device__ __forceinline__ bool col_active(const ColLevel& L, int m) { return !L.act || L.act[m] != 0; }

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
// ghost copies.  A warp takes NL consecutive lines of a row per step (they
// share horizontal neighbours, and the per-lane factors are read once for
// all of them); MINB is the occupancy the register budget is set for.
template <int M, int NL, int MINB>
__global__ void __launch_bounds__(32 * kColWarps, MINB) k_col_sweep(ColLevel L, int color,
                                                                    const float* __restrict__ fac) {
  constexpr int NF = col_fac_floats(M);
  constexpr int N = 32 * M;
  __shared__ float sf[NF];
  __shared__ float sy[kColWarps][NL][N + M];
  for (int q = threadIdx.x; q < NF; q += blockDim.x) sf[q] = fac[q];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float* Fap = sf;
  const float* Frbp = sf + (M - 1) * 32;
  const float* Fsup = sf + 2 * (M - 1) * 32;
  const float* FL = sf + 3 * (M - 1) * 32;
  const float* FR = sf + 4 * (M - 1) * 32;
  const float* Fg = sf + 5 * (M - 1) * 32;
  const int pairs = (L.nx + 1) >> 1;
  const int64_t nlines = (int64_t)pairs * L.ny;  // of one member
  const int64_t ntot = nlines * L.nm;
  const int64_t CS = L.CS, XC = (int64_t)L.X * L.CS;
  const float a1 = L.a1, a2 = L.a2, a3 = L.a3, a4 = L.a4;
  const float c5b = L.cz5[1], c6t = L.cz6[L.nz];  // row 0 to its k=1 ghost, row n-1 to k=Z
  for (int64_t t0 = ((int64_t)blockIdx.x * kColWarps + warp) * NL; t0 < ntot;
       t0 += (int64_t)gridDim.x * kColWarps * NL) {
    int64_t c0[NL];
    bool on[NL];
    int ii[NL], jj[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      const int64_t tt = t0 + l;
      const int m = L.nm == 1 ? 0 : (int)(tt / nlines);
      const int64_t t = tt - (int64_t)m * nlines;
      const int j = 2 + (int)(t / pairs);
      const int i0 = 2 + 2 * (int)(t % pairs);
      const int i = i0 + ((color + i0 + j) & 1);
      on[l] = tt < ntot && i <= L.nx + 1 && col_active(L, m);  // uniform across the warp
      ii[l] = i;
      jj[l] = j;
      c0[l] = on[l] ? m * L.ms + col_cell(L, i, j, 2) : 0;  // row 0
    }
    const float* __restrict__ P = L.phi;
    const float* __restrict__ S = L.src;
    float y[NL][M];
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      float v[M];
      if (on[l]) {
#pragma unroll
        for (int q = 0; q < M; ++q) {
          const int64_t c = c0[l] + lane + 32 * q;
          v[q] = S[c] - (a1 * P[c - CS] + a2 * P[c + CS] + a3 * P[c - XC] + a4 * P[c + XC]);
        }
        if (lane == 0) v[0] -= c5b * P[c0[l] - 1];
        if (lane == 31) v[M - 1] -= c6t * P[c0[l] + N];
      } else {
#pragma unroll
        for (int q = 0; q < M; ++q) v[q] = 0.f;
      }
      // row order -> segment order (lane s: rows s*M .. s*M+M-1)
#pragma unroll
      for (int q = 0; q < M; ++q) sy[warp][l][col_pad(lane + 32 * q)] = v[q];
    }
    __syncwarp();
#pragma unroll
    for (int l = 0; l < NL; ++l)
#pragma unroll
      for (int w = 0; w < M; ++w) y[l][w] = sy[warp][l][col_pad(lane * M + w)];
    __syncwarp();
    // inner rows 0..M-2: local solution with both separators at zero
    float g[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) g[l] = y[l][0];
#pragma unroll
    for (int w = 1; w < M - 1; ++w) {
      const float a = Fap[w * 32 + lane];
#pragma unroll
      for (int l = 0; l < NL; ++l) {
        g[l] = y[l][w] + a * g[l];
        y[l][w] = g[l];
      }
    }
    {
      const float r = Frbp[(M - 2) * 32 + lane];
#pragma unroll
      for (int l = 0; l < NL; ++l) {
        g[l] = g[l] * r;
        y[l][M - 2] = g[l];
      }
    }
#pragma unroll
    for (int w = M - 3; w >= 0; --w) {
      const float c = Fsup[w * 32 + lane], r = Frbp[w * 32 + lane];
#pragma unroll
      for (int l = 0; l < NL; ++l) {
        g[l] = (y[l][w] - c * g[l]) * r;
        y[l][w] = g[l];
      }
    }
    // separator system across the lanes
    const float sub_h = Fg[lane], sup_h = Fg[32 + lane];
    float h[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      const float ynext = __shfl_down_sync(kFull, y[l][0], 1);
      h[l] = y[l][M - 1] - sub_h * y[l][M - 2] - (lane < 31 ? sup_h * ynext : 0.f);
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const int st = 1 << q;
      const float al = Fg[(2 + q) * 32 + lane], ga = Fg[(7 + q) * 32 + lane];
#pragma unroll
      for (int l = 0; l < NL; ++l) {
        const float up = __shfl_up_sync(kFull, h[l], st);
        const float dn = __shfl_down_sync(kFull, h[l], st);
        h[l] = h[l] + al * up + ga * dn;
      }
    }
    float xs[NL], xprev[NL];
    {
      const float rb = Fg[12 * 32 + lane];
#pragma unroll
      for (int l = 0; l < NL; ++l) {
        xs[l] = h[l] * rb;
        xprev[l] = __shfl_up_sync(kFull, xs[l], 1);  // lane 0: L = 0
      }
    }
#pragma unroll
    for (int w = 0; w < M - 1; ++w) {
      const float fl = FL[w * 32 + lane], fr = FR[w * 32 + lane];
#pragma unroll
      for (int l = 0; l < NL; ++l) y[l][w] = y[l][w] + fl * xprev[l] + fr * xs[l];
    }
#pragma unroll
    for (int l = 0; l < NL; ++l) y[l][M - 1] = xs[l];
    // segment order -> row order
#pragma unroll
    for (int l = 0; l < NL; ++l)
#pragma unroll
      for (int w = 0; w < M; ++w) sy[warp][l][col_pad(lane * M + w)] = y[l][w];
    __syncwarp();
    float* __restrict__ Pw = L.phi;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      float v[M];
#pragma unroll
      for (int q = 0; q < M; ++q) v[q] = sy[warp][l][col_pad(lane + 32 * q)];
      if (!on[l]) continue;
      int d0 = kNoImage, d1 = kNoImage, d2 = kNoImage;
      if (L.img) {
        const int* im = L.img + 3 * ((ii[l] - 2) + (int64_t)L.nx * (jj[l] - 2));
        d0 = im[0];
        d1 = im[1];
        d2 = im[2];
      }
      const bool h0 = d0 != kNoImage, h1 = d1 != kNoImage, h2 = d2 != kNoImage;
      const int64_t o0 = h0 ? (int64_t)d0 * CS : 0, o1 = h1 ? (int64_t)d1 * CS : 0,
                    o2 = h2 ? (int64_t)d2 * CS : 0;
#pragma unroll
      for (int q = 0; q < M; ++q) col_put(Pw, c0[l] + lane + 32 * q, v[q], o0, o1, o2, h0, h1, h2);
      // z ghosts of the column and of its images
      const float r0 = __shfl_sync(kFull, v[0], 0);
      const float rn = __shfl_sync(kFull, v[M - 1], 31);
      if (lane == 0 || lane == 31) {
        const int code = lane == 0 ? L.z1 : L.zZ;
        const float gv = code == 0 ? 0.f : (code == 1 ? r0 : rn);
        col_put(Pw, lane == 0 ? c0[l] - 1 : c0[l] + N, gv, o0, o1, o2, h0, h1, h2);
      }
    }
    __syncwarp();
  }
}

// ------------------------------------------- register-factor variant
// The same sweep with the line-independent factors held in registers for
// the life of the warp (5(M-1)+13 per lane: 86 at M = 16) instead of being
// read from shared memory for every line, which takes about a third of the
// L1/shared-memory wavefronts of a line away.  One block of kColWarps warps
// per SM, persistent: each warp walks its lines with a grid stride and,
// before solving one, asks L2 for the five source columns of the next
// (prefetch.global.L2), so their loads are L2 hits when it gets there.
template <int M>
__global__ void __launch_bounds__(32 * kColWarps, 1) k_col_sweep_rf(ColLevel L, int color,
                                                                   const float* __restrict__ fac) {
  constexpr int N = 32 * M;
  constexpr int W = M > 1 ? M - 1 : 1;
  __shared__ float sy[kColWarps][N + M];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float Fap[W], Frbp[W], Fsup[W], FL[W], FR[W];
#pragma unroll
  for (int w = 0; w < M - 1; ++w) {
    Fap[w] = fac[w * 32 + lane];
    Frbp[w] = fac[((M - 1) + w) * 32 + lane];
    Fsup[w] = fac[(2 * (M - 1) + w) * 32 + lane];
    FL[w] = fac[(3 * (M - 1) + w) * 32 + lane];
    FR[w] = fac[(4 * (M - 1) + w) * 32 + lane];
  }
  const float* Fg = fac + 5 * (M - 1) * 32;
  const float sub_h = Fg[lane], sup_h = Fg[32 + lane], rb = Fg[12 * 32 + lane];
  float al[5], ga[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    al[q] = Fg[(2 + q) * 32 + lane];
    ga[q] = Fg[(7 + q) * 32 + lane];
  }
  const int pairs = (L.nx + 1) >> 1;
  const int64_t nlines = (int64_t)pairs * L.ny;  // of one member
  const int64_t ntot = nlines * L.nm;
  const int64_t CS = L.CS, XC = (int64_t)L.X * L.CS;
  const float a1 = L.a1, a2 = L.a2, a3 = L.a3, a4 = L.a4;
  const float c5b = L.cz5[1], c6t = L.cz6[L.nz];
  const int64_t stride = (int64_t)gridDim.x * kColWarps;
  // line tt of the batch: member m, column (i, j); base = m's offset
  auto line = [&](int64_t tt, int& i, int& j, int64_t& base) -> bool {
    const int m = L.nm == 1 ? 0 : (int)(tt / nlines);
    const int64_t t = tt - (int64_t)m * nlines;
    j = 2 + (int)(t / pairs);
    const int i0 = 2 + 2 * (int)(t % pairs);
    i = i0 + ((color + i0 + j) & 1);
    base = m * L.ms;
    return tt < ntot && i <= L.nx + 1 && col_active(L, m);
  };
  float* ys = sy[warp];
  for (int64_t t = (int64_t)blockIdx.x * kColWarps + warp; t < ntot; t += stride) {
    int i, j;
    int64_t mb;
    const bool on = line(t, i, j, mb);
    {
      int in, jn;
      int64_t nb;
      if (line(t + stride, in, jn, nb)) {
        const int64_t cn = nb + col_cell(L, in, jn, 2);
        // the 5 x M 128-byte lines of the next line's source columns
        for (int q = lane; q < 5 * M; q += 32) {
          const int a = q / M, r = (q - a * M) * 32;
          const float* base = a == 0 ? L.src + cn
                                     : L.phi + cn + (a == 1 ? -CS : a == 2 ? CS : a == 3 ? -XC : XC);
          asm volatile("prefetch.global.L2 [%0];\n" ::"l"(base + r));
        }
      }
    }
    if (!on) continue;  // uniform across the warp
    const int64_t c0 = mb + col_cell(L, i, j, 2);
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
#pragma unroll
    for (int q = 0; q < M; ++q) ys[col_pad(lane + 32 * q)] = v[q];
    __syncwarp();
    float y[M];
#pragma unroll
    for (int w = 0; w < M; ++w) y[w] = ys[col_pad(lane * M + w)];
    __syncwarp();
    float g = y[0];
#pragma unroll
    for (int w = 1; w < M - 1; ++w) {
      g = y[w] + Fap[w] * g;
      y[w] = g;
    }
    if (M > 1) {
      float x = g * Frbp[W - 1];
      y[W - 1] = x;
#pragma unroll
      for (int w = M - 3; w >= 0; --w) {
        x = (y[w] - Fsup[w] * x) * Frbp[w];
        y[w] = x;
      }
    }
    const float ynext = __shfl_down_sync(kFull, y[0], 1);
    float h = y[M - 1] - sub_h * (M > 1 ? y[W - 1] : 0.f) - (lane < 31 ? sup_h * ynext : 0.f);
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const int st = 1 << q;
      const float up = __shfl_up_sync(kFull, h, st);
      const float dn = __shfl_down_sync(kFull, h, st);
      h = h + al[q] * up + ga[q] * dn;
    }
    const float xs = h * rb;
    const float xprev = __shfl_up_sync(kFull, xs, 1);
#pragma unroll
    for (int w = 0; w < M - 1; ++w) y[w] = y[w] + FL[w] * xprev + FR[w] * xs;
    y[M - 1] = xs;
#pragma unroll
    for (int w = 0; w < M; ++w) ys[col_pad(lane * M + w)] = y[w];
    __syncwarp();
#pragma unroll
    for (int q = 0; q < M; ++q) v[q] = ys[col_pad(lane + 32 * q)];
    int d0 = kNoImage, d1 = kNoImage, d2 = kNoImage;
    if (L.img) {
      const int* im = L.img + 3 * ((i - 2) + (int64_t)L.nx * (j - 2));
      d0 = im[0];
      d1 = im[1];
      d2 = im[2];
    }
    const bool h0 = d0 != kNoImage, h1 = d1 != kNoImage, h2 = d2 != kNoImage;
    const int64_t o0 = h0 ? (int64_t)d0 * CS : 0, o1 = h1 ? (int64_t)d1 * CS : 0, o2 = h2 ? (int64_t)d2 * CS : 0;
    float* __restrict__ Pw = L.phi;
#pragma unroll
    for (int q = 0; q < M; ++q) col_put(Pw, c0 + lane + 32 * q, v[q], o0, o1, o2, h0, h1, h2);
    const float r0 = __shfl_sync(kFull, v[0], 0);
    const float rn = __shfl_sync(kFull, v[M - 1], 31);
    if (lane == 0 || lane == 31) {
      const int code = lane == 0 ? L.z1 : L.zZ;
      const float gv = code == 0 ? 0.f : (code == 1 ? r0 : rn);
      col_put(Pw, lane == 0 ? c0 - 1 : c0 + N, gv, o0, o1, o2, h0, h1, h2);
    }
    __syncwarp();
  }
}

// ------------------------------------------------ TMA-staged variant
// The same sweep with the line's five source columns (f of the line, phi of
// its four horizontal neighbours: 2 KB each at nz = 512) brought into
// shared memory by 1-D bulk copies (cp.async.bulk, this GPU's own memory,
// no multicast) that complete on an mbarrier.  Each warp double-buffers:
// while it solves one line, the copies of its next line are in flight, so
// the loads need no registers and no load instructions of the warp.  Every
// wait is bounded: after kColWaitLimit polls the kernel records the timeout
// in *err (host-mapped), waits a bounded time more for its copies and
// returns.
constexpr int kColTmaWarps = 4;
constexpr int kColWaitLimit = 1 << 20;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
  for (int it = 0; it < kColWaitLimit; ++it)
    if (mbar_try(bar, parity)) return true;
  return false;
}

template <int M>
__host__ __device__ constexpr size_t col_tma_smem(int warps) {
  // per warp: 2 buffers x 5 columns x N floats, the transpose row, then
  // the factors, then two mbarriers per warp
  return ((size_t)warps * (10 * 32 * M + 33 * M) + col_fac_floats(M)) * sizeof(float) + 16 * warps + 16;
}

template <int M>
__global__ void __launch_bounds__(32 * kColTmaWarps, 2) k_col_sweep_tma(ColLevel L, int color,
                                                                        const float* __restrict__ fac,
                                                                        int* err) {
  constexpr int NF = col_fac_floats(M);
  constexpr int N = 32 * M;
  extern __shared__ __align__(128) float csm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* stage = csm + (size_t)warp * 10 * N;                    // [buf][5][N]
  float* ys = csm + (size_t)kColTmaWarps * 10 * N + (size_t)warp * (N + M);
  float* sf = csm + (size_t)kColTmaWarps * (10 * N + N + M);
  uint64_t* bars = reinterpret_cast<uint64_t*>(
      (reinterpret_cast<uintptr_t>(sf + NF) + 15) & ~(uintptr_t)15);
  for (int q = threadIdx.x; q < NF; q += blockDim.x) sf[q] = fac[q];
  if (lane == 0) {
    for (int b = 0; b < 2; ++b)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bars[2 * warp + b])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  const float* Fap = sf;
  const float* Frbp = sf + (M - 1) * 32;
  const float* Fsup = sf + 2 * (M - 1) * 32;
  const float* FL = sf + 3 * (M - 1) * 32;
  const float* FR = sf + 4 * (M - 1) * 32;
  const float* Fg = sf + 5 * (M - 1) * 32;
  const int pairs = (L.nx + 1) >> 1;
  const int64_t nlines = (int64_t)pairs * L.ny;  // of one member
  const int64_t ntot = nlines * L.nm;
  const int64_t CS = L.CS, XC = (int64_t)L.X * L.CS;
  const float a1 = L.a1, a2 = L.a2, a3 = L.a3, a4 = L.a4;
  const float c5b = L.cz5[1], c6t = L.cz6[L.nz];
  const int64_t stride = (int64_t)gridDim.x * kColTmaWarps;
  // line tt of the batch: member m (base = its offset), column (i, j);
  // the lines of inactive members are copied in too (the buffer parity
  // below counts every line) but not solved
  auto line = [&](int64_t tt, int& i, int& j, int64_t& base, bool& act) -> bool {
    const int m = L.nm == 1 ? 0 : (int)(tt / nlines);
    const int64_t t = tt - (int64_t)m * nlines;
    j = 2 + (int)(t / pairs);
    const int i0 = 2 + 2 * (int)(t % pairs);
    i = i0 + ((color + i0 + j) & 1);
    base = m * L.ms;
    act = tt < ntot && col_active(L, m);
    return tt < ntot && i <= L.nx + 1;
  };
  // lane 0: the five source columns of line t into buffer b
  auto issue = [&](int64_t t, int b) {
    int i, j;
    int64_t base;
    bool act;
    if (!line(t, i, j, base, act)) return;
    const int64_t c0 = base + col_cell(L, i, j, 2);
    const unsigned bar = smem_u32(&bars[2 * warp + b]);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(5 * N * 4) : "memory");
    const float* src[5] = {L.src + c0, L.phi + c0 - CS, L.phi + c0 + CS, L.phi + c0 - XC, L.phi + c0 + XC};
#pragma unroll
    for (int a = 0; a < 5; ++a)
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
              smem_u32(stage + (size_t)(b * 5 + a) * N)),
          "l"(src[a]), "r"(N * 4), "r"(bar)
          : "memory");
  };
  // (every line is valid for even nx, which the launcher requires, so the
  // u-th line of a warp is the (u/2)-th use of buffer u%2: parity u/2 % 2)
  int64_t t = (int64_t)blockIdx.x * kColTmaWarps + warp;
  if (lane == 0) issue(t, 0);
  int u = 0;
  bool ok = true;
  for (; t < ntot; ++u, t += stride) {
    const int b = u & 1;
    if (lane == 0) issue(t + stride, b ^ 1);
    int i, j;
    int64_t mb;
    bool act;
    (void)line(t, i, j, mb, act);
    if (!mbar_wait(smem_u32(&bars[2 * warp + b]), (unsigned)((u >> 1) & 1))) {
      ok = false;
      break;
    }
    if (!act) {  // uniform across the warp
      __syncwarp();
      continue;
    }
    const int64_t c0 = mb + col_cell(L, i, j, 2);
    const float* sb = stage + (size_t)b * 5 * N;
    float v[M];
#pragma unroll
    for (int q = 0; q < M; ++q) {
      const int r = lane + 32 * q;
      v[q] = sb[r] - (a1 * sb[N + r] + a2 * sb[2 * N + r] + a3 * sb[3 * N + r] + a4 * sb[4 * N + r]);
    }
    if (lane == 0) v[0] -= c5b * L.phi[c0 - 1];
    if (lane == 31) v[M - 1] -= c6t * L.phi[c0 + N];
#pragma unroll
    for (int q = 0; q < M; ++q) ys[col_pad(lane + 32 * q)] = v[q];
    __syncwarp();
    float y[M];
#pragma unroll
    for (int w = 0; w < M; ++w) y[w] = ys[col_pad(lane * M + w)];
    __syncwarp();
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
    const float ynext = __shfl_down_sync(kFull, y[0], 1);
    float h = y[M - 1] - Fg[lane] * y[M - 2] - (lane < 31 ? Fg[32 + lane] * ynext : 0.f);
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const int st = 1 << q;
      const float up = __shfl_up_sync(kFull, h, st);
      const float dn = __shfl_down_sync(kFull, h, st);
      h = h + Fg[(2 + q) * 32 + lane] * up + Fg[(7 + q) * 32 + lane] * dn;
    }
    const float xs = h * Fg[12 * 32 + lane];
    const float xprev = __shfl_up_sync(kFull, xs, 1);
#pragma unroll
    for (int w = 0; w < M - 1; ++w) y[w] = y[w] + FL[w * 32 + lane] * xprev + FR[w * 32 + lane] * xs;
    y[M - 1] = xs;
#pragma unroll
    for (int w = 0; w < M; ++w) ys[col_pad(lane * M + w)] = y[w];
    __syncwarp();
#pragma unroll
    for (int q = 0; q < M; ++q) v[q] = ys[col_pad(lane + 32 * q)];
    int d0 = kNoImage, d1 = kNoImage, d2 = kNoImage;
    if (L.img) {
      const int* im = L.img + 3 * ((i - 2) + (int64_t)L.nx * (j - 2));
      d0 = im[0];
      d1 = im[1];
      d2 = im[2];
    }
    const bool h0 = d0 != kNoImage, h1 = d1 != kNoImage, h2 = d2 != kNoImage;
    const int64_t o0 = h0 ? (int64_t)d0 * CS : 0, o1 = h1 ? (int64_t)d1 * CS : 0, o2 = h2 ? (int64_t)d2 * CS : 0;
    float* __restrict__ Pw = L.phi;
#pragma unroll
    for (int q = 0; q < M; ++q) col_put(Pw, c0 + lane + 32 * q, v[q], o0, o1, o2, h0, h1, h2);
    const float r0 = __shfl_sync(kFull, v[0], 0);
    const float rn = __shfl_sync(kFull, v[M - 1], 31);
    if (lane == 0 || lane == 31) {
      const int code = lane == 0 ? L.z1 : L.zZ;
      const float gv = code == 0 ? 0.f : (code == 1 ? r0 : rn);
      col_put(Pw, lane == 0 ? c0 - 1 : c0 + N, gv, o0, o1, o2, h0, h1, h2);
    }
    __syncwarp();  // every lane is done with buffer b before it is refilled
  }
  if (!ok) {
    if (lane == 0) *reinterpret_cast<volatile int*>(err) = 1;
    // bounded wait for this warp's copies still in flight (line t in
    // buffer u%2, and line t+stride in the other buffer if it exists),
    // then return
    (void)mbar_wait(smem_u32(&bars[2 * warp + (u & 1)]), (unsigned)((u >> 1) & 1));
    if (t + stride < ntot)
      (void)mbar_wait(smem_u32(&bars[2 * warp + ((u + 1) & 1)]), (unsigned)(((u + 1) >> 1) & 1));
  }
}

// Residuals f - A phi of fine cells (i,j,k..k+3) (k-2 a multiple of 4, so
// the four cells are one aligned 16-byte vector), in fine_resid's order.
__device__ __forceinline__ float4 col_resid4(const ColLevel& F, int i, int j, int k) {
  const int64_t c = col_cell(F, i, j, k);
  const float* __restrict__ p = F.phi;
  const int64_t CS = F.CS, XC = (int64_t)F.X * F.CS;
  const float4 C = *reinterpret_cast<const float4*>(p + c);
  const float4 W = *reinterpret_cast<const float4*>(p + c - CS);
  const float4 E = *reinterpret_cast<const float4*>(p + c + CS);
  const float4 S = *reinterpret_cast<const float4*>(p + c - XC);
  const float4 N = *reinterpret_cast<const float4*>(p + c + XC);
  const float4 Fv = *reinterpret_cast<const float4*>(F.src + c);
  const float pm = p[c - 1], pp = p[c + 4];
  const float cv[4] = {C.x, C.y, C.z, C.w}, wv[4] = {W.x, W.y, W.z, W.w}, ev[4] = {E.x, E.y, E.z, E.w};
  const float sv[4] = {S.x, S.y, S.z, S.w}, nv[4] = {N.x, N.y, N.z, N.w}, fv[4] = {Fv.x, Fv.y, Fv.z, Fv.w};
  const float dv[4] = {pm, C.x, C.y, C.z}, uv[4] = {C.y, C.z, C.w, pp};
  float r[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int kq = k + q;
    const float diag = -(F.a1 + F.a2 + F.a3 + F.a4 + F.dz5[kq - 1] + F.dz6[kq - 1]);
    float acc = F.a1 * wv[q];
    acc = acc + F.a2 * ev[q];
    acc = acc + F.a3 * sv[q];
    acc = acc + F.a4 * nv[q];
    acc = acc + F.cz5[kq - 1] * dv[q];
    acc = acc + F.cz6[kq - 1] * uv[q];
    acc = acc + diag * cv[q];
    r[q] = fv[q] - acc;
  }
  return make_float4(r[0], r[1], r[2], r[3]);
}

__device__ __forceinline__ float4 f4add(float4 a, float4 b) {
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__device__ __forceinline__ float4 f4scale(float s, float4 a) {
  return make_float4(s * a.x, s * a.y, s * a.z, s * a.w);
}

constexpr int kColXferThreads = 256;

// Grid of the transfer kernels: x runs over (column of a row, 4-row chunk)
// with the chunk fastest, y over the rows of columns, z over the members of
// a batch; 32-bit indices (a row holds far fewer than 2^32 chunks).

// mg_restr's x/y variants (z is not coarsened): coarse f of interior cells
// (ic,jc,k..k+3) from the residuals of their children, in restrict_value's
// order.  One thread per coarse column and 4-row chunk; the caller zeroes
// coarse phi.
template <int CD>
__global__ void __launch_bounds__(kColXferThreads) k_col_restrict(ColLevel Fb, ColLevel Cb) {
  const int m = blockIdx.z;
  if (!col_active(Cb, m)) return;
  const unsigned nch = (unsigned)Cb.nz >> 2;
  const unsigned t = blockIdx.x * kColXferThreads + threadIdx.x;
  if (t >= (unsigned)Cb.nx * nch) return;
  constexpr bool cx = CD & 1, cy = CD & 2;
  const ColLevel F = col_member(Fb, m);
  const ColLevel C = col_member(Cb, m);
  const unsigned q = t / nch;
  const int ch = (int)(t - q * nch);
  const int ic = 2 + (int)q, jc = 2 + (int)blockIdx.y;
  const int k = 2 + 4 * ch;
  const int i = cx ? 2 * ic - 2 : ic;
  const int j = cy ? 2 * jc - 2 : jc;
  float4 v;
  if constexpr (cx && cy) {
    float4 s = col_resid4(F, i, j, k);
    s = f4add(s, col_resid4(F, i + 1, j, k));
    s = f4add(s, col_resid4(F, i, j + 1, k));
    s = f4add(s, col_resid4(F, i + 1, j + 1, k));
    v = f4scale(0.25f, s);
  } else if constexpr (cx) {
    v = f4scale(0.5f, f4add(col_resid4(F, i, j, k), col_resid4(F, i + 1, j, k)));
  } else {
    v = f4scale(0.5f, f4add(col_resid4(F, i, j, k), col_resid4(F, i, j + 1, k)));
  }
  *reinterpret_cast<float4*>(C.src + col_cell(C, ic, jc, k)) = v;
}

// Adds the correction chunk corr to rows k..k+3 of fine column (i,j) and
// writes the sum to the column, to its image columns and, from the first
// and last chunks, to its z ghosts (the boundary pass of the row-major
// cycle).
__device__ __forceinline__ void col_prolong_store(const ColLevel& F, int i, int j, int k, int ch, int nch,
                                                  float4 corr) {
  const int64_t c = col_cell(F, i, j, k);
  float* __restrict__ P = F.phi;
  const float4 old = *reinterpret_cast<const float4*>(P + c);
  const float4 v = f4add(old, corr);
  int d0 = kNoImage, d1 = kNoImage, d2 = kNoImage;
  if (F.img) {
    const int* im = F.img + 3 * ((i - 2) + (int64_t)F.nx * (j - 2));
    d0 = im[0];
    d1 = im[1];
    d2 = im[2];
  }
  const int64_t o0 = (int64_t)d0 * F.CS, o1 = (int64_t)d1 * F.CS, o2 = (int64_t)d2 * F.CS;
  *reinterpret_cast<float4*>(P + c) = v;
  if (d0 != kNoImage) *reinterpret_cast<float4*>(P + c + o0) = v;
  if (d1 != kNoImage) *reinterpret_cast<float4*>(P + c + o1) = v;
  if (d2 != kNoImage) *reinterpret_cast<float4*>(P + c + o2) = v;
  // z ghosts: the first chunk writes the ghosts that copy row k = 2 or
  // are zero, the last chunk those that copy row k = nz+1
  const bool h0 = d0 != kNoImage, h1 = d1 != kNoImage, h2 = d2 != kNoImage;
  const int64_t g1 = c - (k - 1), gZ = c + (F.nz + 2 - k);
  if (ch == 0) {
    if (F.z1 != 2) col_put(P, g1, F.z1 == 1 ? v.x : 0.f, o0, o1, o2, h0, h1, h2);
    if (F.zZ != 2) col_put(P, gZ, F.zZ == 1 ? v.x : 0.f, o0, o1, o2, h0, h1, h2);
  }
  if (ch == nch - 1) {
    if (F.z1 == 2) col_put(P, g1, v.w, o0, o1, o2, h0, h1, h2);
    if (F.zZ == 2) col_put(P, gZ, v.w, o0, o1, o2, h0, h1, h2);
  }
}

// mg_cor's x/y variants for the fine interior, in prolong_corr's order,
// with the ghost copies of the updated cells written alongside.  Fine
// columns i = 2g+1 and 2g+2 both interpolate between coarse columns g+1
// and g+2 (weights 3:1 and 1:3) when x is coarsened, likewise in y: one
// thread per 4-row chunk of such a group of up to 2x2 fine columns (the
// ghost columns i = 1, nx+2 / j = 1, ny+2 of the edge groups are skipped)
// loads the four coarse chunks once.
template <int CD>
__global__ void __launch_bounds__(kColXferThreads) k_col_prolong(ColLevel Fb, ColLevel Cb) {
  const int m = blockIdx.z;
  if (!col_active(Fb, m)) return;
  constexpr bool cx = CD & 1, cy = CD & 2;
  const unsigned nch = (unsigned)Fb.nz >> 2;
  const unsigned gxn = cx ? (unsigned)(Fb.nx >> 1) + 1u : (unsigned)Fb.nx;  // groups per row
  const unsigned t = blockIdx.x * kColXferThreads + threadIdx.x;
  if (t >= gxn * nch) return;
  const ColLevel F = col_member(Fb, m);
  const ColLevel C = col_member(Cb, m);
  const unsigned q = t / nch;
  const int ch = (int)(t - q * nch);
  const int gx = (int)q, gy = (int)blockIdx.y;
  const int k = 2 + 4 * ch;
  const int i0 = cx ? 2 * gx + 1 : gx + 2, j0 = cy ? 2 * gy + 1 : gy + 2;
  const int ic = cx ? gx + 1 : i0, jc = cy ? gy + 1 : j0;
  const float* __restrict__ pc = C.phi + col_cell(C, ic, jc, k);
  const int64_t ox = C.CS, oy = (int64_t)C.X * C.CS;
  const float4 c00 = *reinterpret_cast<const float4*>(pc);
  if constexpr (cx && cy) {
    const float4 c10 = *reinterpret_cast<const float4*>(pc + ox);
    const float4 c01 = *reinterpret_cast<const float4*>(pc + oy);
    const float4 c11 = *reinterpret_cast<const float4*>(pc + ox + oy);
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int j = j0 + b;
      if (j < 2 || j > F.ny + 1) continue;
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        const int i = i0 + a;
        if (i < 2 || i > F.nx + 1) continue;
        const float wx0 = (i & 1) ? 3.f : 1.f, wx1 = (i & 1) ? 1.f : 3.f;
        const float wy0 = (j & 1) ? 3.f : 1.f, wy1 = (j & 1) ? 1.f : 3.f;
        const float w00 = wx0 * wy0, w10 = wx1 * wy0, w01 = wx0 * wy1, w11 = wx1 * wy1;
        auto one = [&](float p, float r, float u, float d) {
          float s = w00 * p;
          s = s + w10 * r;
          s = s + w01 * u;
          s = s + w11 * d;
          return s / 16.f;
        };
        const float4 corr = make_float4(one(c00.x, c10.x, c01.x, c11.x), one(c00.y, c10.y, c01.y, c11.y),
                                        one(c00.z, c10.z, c01.z, c11.z), one(c00.w, c10.w, c01.w, c11.w));
        col_prolong_store(F, i, j, k, ch, (int)nch, corr);
      }
    }
  } else {
    const float4 c1 = *reinterpret_cast<const float4*>(pc + (cx ? ox : oy));
    constexpr int n2 = 2;
#pragma unroll
    for (int a = 0; a < n2; ++a) {
      const int i = cx ? i0 + a : i0, j = cx ? j0 : j0 + a;
      if (cx ? (i < 2 || i > F.nx + 1) : (j < 2 || j > F.ny + 1)) continue;
      const int par = cx ? (i & 1) : (j & 1);
      const float w0 = par ? 3.f : 1.f, w1 = par ? 1.f : 3.f;
      const float4 corr = make_float4((w0 * c00.x + w1 * c1.x) / 4.f, (w0 * c00.y + w1 * c1.y) / 4.f,
                                      (w0 * c00.z + w1 * c1.z) / 4.f, (w0 * c00.w + w1 * c1.w) / 4.f);
      col_prolong_store(F, i, j, k, ch, (int)nch, corr);
    }
  }
}

}  // namespace anel
