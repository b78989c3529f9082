// Density matrix by trace-correcting purification, inside one CTA.
//
// The SCF step needs P = 2 C_occ C_occ^T, the projector onto the nocc lowest eigenstates of F
// -- the aufbau density the reference builds from LAPACK's eigenvectors
// (scfcalculation.cpp:94-110, densitymatrix.cpp:40-56).  The projector is also the limit of
// the TC2 recursion (A. M. N. Niklasson, Phys. Rev. B 66, 155115 (2002)):
//   X_0 = (e_max I - F) / (e_max - e_min)     (spectrum mapped into [0, 1], order reversed)
//   X_{k+1} = X_k^2          if |tr(X_k^2) - nocc| < |2 tr(X_k) - tr(X_k^2) - nocc|
//           = 2 X_k - X_k^2  otherwise
// with e_min, e_max Gershgorin bounds.  Each step is one symmetric matrix square, so the
// eigensolve becomes ~20 dense products, run on the FP64 tensor-core path (DMMA m8n8k4).
// tr(X^2) = ||X||_F^2 for symmetric X, so the branch of the next step is known from the
// element sums of the current one, before its product starts.
//
// X lives in shared memory: n16 x n16 (nao rounded up to 16, zero padding, which stays zero),
// row stride n16 + 4 doubles (8 rows x 4 columns of a fragment load then fall in distinct banks
// within each half-warp phase).  The product's lower triangle is tiled in 16 x 16 super-tiles,
// dealt round-robin to the warps; each warp keeps its accumulators in registers until every
// warp has finished reading X, then writes the new X (lower triangle and its mirror) in place.
//
// Convergence: tr(X - X^2) = sum lambda (1 - lambda) is the idempotency error; once it is
// below kPurifyIdem the eigenvalues are within ~1e-8 of 0 or 1 and kPurifyTail more steps
// (quadratic) take them to rounding level.  A result is accepted only if tr(X) = nocc; a
// vanishing HOMO-LUMO gap (no convergence within kPurifyMaxIter) or any non-finite value
// reports failure, and the caller diagonalises instead.
#pragma once
#include "scf_block.cuh"

namespace sgb {

constexpr int kPurifyMaxIter = 64;
constexpr double kPurifyIdem = 1e-8;
constexpr int kPurifyTail = 2;
constexpr double kPurifyTraceTol = 1e-6;
constexpr int kPurifyMaxN16 = 160;  // largest padded order held in one CTA's shared memory
// Mixed precision (grid path): FP32 products until tr(X - X^2) falls below this, FP64 after.
constexpr double kPurifyMixedSwitch = 1e-3;

__host__ __device__ inline int purify_n16(int n) { return (n + 15) & ~15; }
__host__ __device__ inline int purify_ld(int n) { return purify_n16(n) + 4; }
__host__ __device__ inline size_t purify_doubles(int n) {
  return (size_t)purify_n16(n) * (size_t)purify_ld(n);
}

// D (8x8, two values per lane) += A (8x4, one per lane) * B (4x8, one per lane).  Lane l holds
// A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4)], D[l/4][2(l%4)+1].
__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// Block-wide sums of two values, identical in every thread (fixed summation order).
template <int NT>
__device__ __forceinline__ void block_sum2(double& a, double& b, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) { red[w] = a; red[16 + w] = b; }
  __syncthreads();
  a = 0.0;
  b = 0.0;
#pragma unroll
  for (int k = 0; k < NT / 32; ++k) { a += red[k]; b += red[16 + k]; }
  __syncthreads();
}

// X_0 from F (row-major n x n, global) and its trace / squared norm.
template <int NT>
__device__ void purify_init(const double* F, int n, double* X, int ld, double* red, double& t1,
                            double& t2) {
  constexpr int NW = NT / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double lo = INFINITY, hi = -INFINITY;
  for (int i = warp; i < n; i += NW) {
    const double* row = F + (int64_t)i * n;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += j == i ? 0.0 : fabs(row[j]);
    s = warp_sum(s);
    const double d = row[i];
    lo = fmin(lo, d - s);
    hi = fmax(hi, d + s);
  }
  hi = block_max<NT>(hi, red);
  lo = -block_max<NT>(-lo, red);
  if (!(hi - lo > 1e-12)) hi = lo + 1.0;  // F a multiple of I (or not finite: caught later)
  const double inv = 1.0 / (hi - lo);
  const int n16 = purify_n16(n);
  double s1 = 0.0, s2 = 0.0;
  for (int t = threadIdx.x; t < n16 * n16; t += NT) {
    const int r = t / n16, c = t - r * n16;
    double v = 0.0;
    if (r < n && c < n) v = ((r == c ? hi : 0.0) - F[(int64_t)r * n + c]) * inv;
    X[r * ld + c] = v;
    if (r == c) s1 += v;
    s2 = fma(v, v, s2);
  }
  block_sum2<NT>(s1, s2, red);
  t1 = s1;
  t2 = s2;
}

// X <- X^2 (sq) or 2X - X^2 (!sq), in place; t1, t2 <- trace and squared norm of the result.
// MAXST: super-tiles per warp (the launch's count rounded up), so the accumulators of smaller
// orders take fewer registers.  Two barriers per step: after the product (every warp has read
// X) and after the write-back (X and the per-warp partial sums complete).  The partial sums
// alternate between two halves of red (buf), so the next step's writes never meet this step's
// reads.
template <int NT, int MAXST>
__device__ __noinline__ void purify_step(double* X, int n16, int ld, bool sq, double* red,
                                         int buf, double& t1, double& t2) {
  constexpr int NW = NT / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, q = lane & 3;
  const int nst = n16 >> 4, cnt = nst * (nst + 1) / 2;
  double acc[MAXST][4][2];
  int rowI[MAXST], rowJ[MAXST];
#pragma unroll
  for (int u = 0; u < MAXST; ++u) {
    int I = 0, J = 0;
    if (warp + u * NW < cnt) tri_inverse(warp + u * NW, I, J);
    rowI[u] = (I * 16 + g) * ld + q;
    rowJ[u] = (J * 16 + g) * ld + q;
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[u][k][0] = acc[u][k][1] = 0.0;
  }
  for (int k0 = 0; k0 < n16; k0 += 4) {
#pragma unroll
    for (int u = 0; u < MAXST; ++u) {
      if (warp + u * NW < cnt) {
        const double a0 = X[rowI[u] + k0], a1 = X[rowI[u] + 8 * ld + k0];
        const double b0 = X[rowJ[u] + k0], b1 = X[rowJ[u] + 8 * ld + k0];
        dmma884(acc[u][0][0], acc[u][0][1], a0, b0);
        if (rowI[u] != rowJ[u]) dmma884(acc[u][1][0], acc[u][1][1], a0, b1);
        dmma884(acc[u][2][0], acc[u][2][1], a1, b0);
        dmma884(acc[u][3][0], acc[u][3][1], a1, b1);
      }
    }
  }
  __syncthreads();  // every warp has read X
  double s1 = 0.0, s2 = 0.0;
#pragma unroll
  for (int u = 0; u < MAXST; ++u) {
    if (warp + u * NW < cnt) {
      int I, J;
      tri_inverse(warp + u * NW, I, J);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int r = I * 16 + (k >> 1) * 8 + g;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int c = J * 16 + (k & 1) * 8 + 2 * q + e;
          if (r >= c) {
            const double x2 = acc[u][k][e];
            const double v = sq ? x2 : fma(2.0, X[r * ld + c], -x2);
            X[r * ld + c] = v;
            if (r != c) X[c * ld + r] = v;
            if (r == c) s1 += v;
            s2 = fma(r == c ? v : 2.0 * v, v, s2);
          }
        }
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  double* part = red + 32 * buf;
  if (lane == 0) { part[warp] = s1; part[16 + warp] = s2; }
  __syncthreads();
  s1 = 0.0;
  s2 = 0.0;
#pragma unroll
  for (int k = 0; k < NW; ++k) { s1 += part[k]; s2 += part[16 + k]; }
  t1 = s1;
  t2 = s2;
}

// Purifies F (row-major n x n in global memory) into X = P / 2 in shared memory.  Returns the
// number of products, or -1 (no convergence, wrong trace or a non-finite value).  red: 64
// doubles.
template <int NT>
__device__ int block_purify(const double* F, int n, int nocc, double* X, double* red) {
  const int ld = purify_ld(n), n16 = purify_n16(n);
  double t1, t2;
  purify_init<NT>(F, n, X, ld, red, t1, t2);
  int tail = -1;
  for (int it = 0; it <= kPurifyMaxIter; ++it) {
    if (!(fabs(t1) < INFINITY) || !(fabs(t2) < INFINITY)) return -1;
    if (tail < 0 && t1 - t2 < kPurifyIdem) tail = kPurifyTail;
    if (tail == 0) return fabs(t1 - (double)nocc) < kPurifyTraceTol ? it : -1;
    if (tail > 0) --tail;
    if (it == kPurifyMaxIter) break;
    const double n_o = (double)nocc;
    const bool sq = fabs(t2 - n_o) < fabs(2.0 * t1 - t2 - n_o);
    constexpr int NW = NT / 32;
    constexpr int kSuper = (kPurifyMaxN16 / 16) * (kPurifyMaxN16 / 16 + 1) / 2;
    const int cnt = (n16 >> 4) * ((n16 >> 4) + 1) / 2;
    const int buf = it & 1;
    if (cnt <= NW)
      purify_step<NT, 1>(X, n16, ld, sq, red, buf, t1, t2);
    else if (cnt <= 2 * NW)
      purify_step<NT, 2>(X, n16, ld, sq, red, buf, t1, t2);
    else if (cnt <= 3 * NW || (kSuper + NW - 1) / NW <= 3)
      purify_step<NT, 3>(X, n16, ld, sq, red, buf, t1, t2);
    else if constexpr (NT >= 256)
      purify_step<NT, (kSuper + NW - 1) / NW>(X, n16, ld, sq, red, buf, t1, t2);
    else
      return -1;  // 128-thread CTAs only take nao <= 64 (at most 10 super-tiles)
  }
  return -1;
}

// P (packed lower triangle) = 2 X.
__device__ inline void purify_density(const double* X, int n, double* P) {
  const int ld = purify_ld(n);
  const int64_t np = tri(n);
  for (int64_t t = threadIdx.x; t < np; t += blockDim.x) {
    int i, j;
    tri_inverse(t, i, j);
    P[t] = 2.0 * X[i * ld + j];
  }
}

}  // namespace sgb
