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
// row stride n16 + 8 doubles (the two rows of a quarter-warp's 16-byte fragment loads fall in
// opposite halves of the banks).  The product's lower triangle is tiled in 16 x 16 super-tiles,
// dealt round-robin to the warps; each warp keeps its accumulators in registers until every
// warp has finished reading X, then writes the new X (lower triangle and its mirror) in place.
//
// Convergence: tr(X - X^2) = sum lambda (1 - lambda) is the idempotency error; once it is
// below kPurifyIdem the eigenvalues are within ~1e-8 of 0 or 1 and kPurifyTail more steps
// (quadratic) take them to rounding level, unless it falls below kPurifyIdemFinal first.  A result is accepted only if tr(X) = nocc; a
// vanishing HOMO-LUMO gap (no convergence within kPurifyMaxIter) or any non-finite value
// reports failure, and the caller diagonalises instead.
#pragma once
#include "scf_block.cuh"

namespace sgb {

constexpr int kPurifyMaxIter = 64;
constexpr double kPurifyIdem = 1e-8;
// Done at once when tr(X - X^2) is below this: every eigenvalue is then within 1e-11 of 0 or 1
// (the tail after kPurifyIdem exists for the case where one side of the spectrum has not been
// squared yet; reaching this bound first saves those products).
constexpr double kPurifyIdemFinal = 1e-11;
constexpr int kPurifyTail = 2;
constexpr double kPurifyTraceTol = 1e-6;
constexpr int kPurifyMaxN16 = 160;  // largest padded order held in one CTA's shared memory
// Mixed precision (grid path): FP32 products until tr(X - X^2) falls below this, FP64 after.
constexpr double kPurifyMixedSwitch = 1e-3;
// The mixed form's FP64 finish (every size that runs the tensor-core phase) ends once
// tr(X - X^2) < kMixedIdemFinal, with no tail.  X is a polynomial in F, so it has F's eigenvectors;
// an eigenvalue lambda_i of X near 0 or 1 is off by about lambda_i (1 - lambda_i), and E_el moves
// by at most 2 sum_i lambda_i (1 - lambda_i) |e_i| <= 2 tr(X - X^2) max |e_i| (e_i: eigenvalues
// of F, |e_i| < 100 eV for H, C, N, O), i.e. 2e-7 eV: well inside the form's 1e-4 eV and below
// the SCF's 1e-6 eV step test.  The 1e-10 this replaced cost one more pair of FP64 products in
// most purifications (148 alkanes of 164-902 AOs in one batch: 528 -> 435 ms).
constexpr double kMixedIdemFinal = 1e-9;

// Spectral bounds.  Gershgorin discs are always valid but loose (about 2.5x the width of the
// spectrum for these Fock matrices), and every doubling of the interval costs TC2 about two
// products.  Above kLanczosMinN a short Lanczos run gives the extreme Ritz values theta and
// residual radii beta_K |s_K| (an eigenvalue of F lies within that radius of each Ritz
// value); the interval theta_min - r_min - kLanczosMargin .. theta_max + r_max + kLanczosMargin,
// clipped to the Gershgorin interval, cut the products by about 20 % on the reference cases
// and held the whole spectrum on every one of them.  Should an eigenvalue still fall outside,
// its trace and idempotency checks fail and the step is diagonalised instead.
constexpr int kLanczosSteps = 8;
constexpr int kLanczosMinN = 32;
constexpr double kLanczosMargin = 1.0;  // eV

// Deterministic start vector with entries in [0.5, 1.5) (not normalised): no symmetry of the
// molecule singles it out, so every symmetry block of F is seen.
__host__ __device__ inline double lanczos_start(int i) {
  uint32_t h = (uint32_t)i * 2654435761u + 12345u;
  h = (h ^ (h >> 15)) * 2246822519u;
  return 0.5 + (double)h * (1.0 / 4294967296.0);
}

// Number of eigenvalues below x of the symmetric tridiagonal (a[0..k), b[0..k-1)): sign
// changes of the leading principal minors p_i = det(T_i - x I) (Sturm), by the three-term
// recurrence -- products only, no division (k <= 8 keeps them far from overflow).
template <int K>
__host__ __device__ inline int sturm_count(const double* a, const double* b, double x) {
  int c = 0;
  double pm = 1.0, p = a[0] - x;
  c += p < 0.0;
#pragma unroll
  for (int i = 1; i < K; ++i) {
    const double pn = (a[i] - x) * p - b[i - 1] * b[i - 1] * pm;
    c += (pn < 0.0) != (p < 0.0);
    pm = p;
    p = pn;
  }
  return c;
}

// Smallest (lowest = true) or largest eigenvalue of the K x K tridiagonal by bisection.
// K is a template parameter so that a, b stay in registers.
template <int K>
__host__ __device__ inline double tridiag_extreme(const double* a, const double* b, bool lowest) {
  double lo = INFINITY, hi = -INFINITY;
#pragma unroll
  for (int i = 0; i < K; ++i) {
    const double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i < K - 1 ? fabs(b[i]) : 0.0);
    lo = fmin(lo, a[i] - r);
    hi = fmax(hi, a[i] + r);
  }
  const int target = lowest ? 1 : K;
#ifdef __CUDA_ARCH__
  // 33-way bisection across the warp: lane l tests lo + (l + 1) (hi - lo) / 33; 8 rounds shrink
  // the interval by 33^8 (every warp of the CTA computes the same result)
  const int lane = threadIdx.x & 31;
  for (int round = 0; round < 8; ++round) {
    const double h = (hi - lo) * (1.0 / 33.0);
    const double x = lo + (lane + 1) * h;
    const unsigned ge = __ballot_sync(0xffffffffu, sturm_count<K>(a, b, x) >= target);
    const int first = ge ? __ffs(ge) - 1 : 32;  // first test point at or above the eigenvalue
    hi = lo + (first + 1) * h;
    lo = lo + first * h;
  }
#else
  for (int it = 0; it < 56; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (sturm_count<K>(a, b, mid) >= target) hi = mid;
    else lo = mid;
  }
#endif
  return 0.5 * (lo + hi);
}

// |last component| of the normalised eigenvector of the tridiagonal for eigenvalue th.
template <int K>
__host__ __device__ inline double tridiag_last(const double* a, const double* b, double th) {
  double xm = 0.0, x = 1.0, nrm = 1.0;
#pragma unroll
  for (int i = 0; i + 1 < K; ++i) {
    const double xn = ((th - a[i]) * x - (i > 0 ? b[i - 1] * xm : 0.0)) / b[i];
    xm = x;
    x = xn;
    nrm += x * x;
  }
  return fabs(x) / sqrt(nrm);
}

// Lanczos-refined bounds from the coefficients of K steps (beta_last = the K-th beta).
template <int K>
__host__ __device__ inline void lanczos_bounds(const double* a, const double* b,
                                               double beta_last, double& lo, double& hi) {
  const double tmin = tridiag_extreme<K>(a, b, true), tmax = tridiag_extreme<K>(a, b, false);
  const double rmin = beta_last * tridiag_last<K>(a, b, tmin);
  const double rmax = beta_last * tridiag_last<K>(a, b, tmax);
  lo = tmin - rmin - kLanczosMargin;
  hi = tmax + rmax + kLanczosMargin;
}

__host__ __device__ inline int purify_n16(int n) { return (n + 15) & ~15; }
__host__ __device__ inline int purify_ld(int n) { return purify_n16(n) + 8; }
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

// X_0 from F (row-major n x n, global) and its trace / squared norm.  F is read once, into the
// X region (row stride ld, zero padding); the Gershgorin sums, the Lanczos products and the
// map to X_0 (in place) then work from shared memory.  lz: 3 n doubles of shared scratch.
template <int NT>
__device__ __noinline__ void purify_init(const double* F, int n, double* X, int ld, double* lz, double* red,
                            double& t1, double& t2) {
  constexpr int NW = NT / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n16 = purify_n16(n);
  for (int t = threadIdx.x; t < n16 * n16; t += NT) {
    const int r = t / n16, c = t - r * n16;
    X[r * ld + c] = (r < n && c < n) ? F[(int64_t)r * n + c] : 0.0;
  }
  __syncthreads();
  double lo = INFINITY, hi = -INFINITY;
  for (int i = warp; i < n; i += NW) {
    const double* row = X + i * ld;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += j == i ? 0.0 : fabs(row[j]);
    s = warp_sum(s);
    const double d = row[i];
    lo = fmin(lo, d - s);
    hi = fmax(hi, d + s);
  }
  hi = block_max<NT>(hi, red);
  lo = -block_max<NT>(-lo, red);
  if (n > kLanczosMinN) {
    double* q = lz;
    double* qp = lz + n;
    double* w = lz + 2 * n;
    double s0 = 0.0;
    for (int i = threadIdx.x; i < n; i += NT) {
      const double v = lanczos_start(i);
      q[i] = v;
      qp[i] = 0.0;
      s0 = fma(v, v, s0);
    }
    const double inv0 = 1.0 / sqrt(block_sum<NT>(s0, red));
    for (int i = threadIdx.x; i < n; i += NT) q[i] *= inv0;
    __syncthreads();
    double al[kLanczosSteps], be[kLanczosSteps];
    double beta = 0.0;
    bool broke = false;  // an invariant subspace: its Ritz values need not bound F's spectrum
#pragma unroll
    for (int k = 0; k < kLanczosSteps; ++k) {
      // w = F q - beta q_prev, two rows per warp at a time; every lane accumulates its rows'
      // q.w and w.w, so one barrier completes both the vector and the sums
      double qw = 0.0, ww = 0.0;
      for (int i = warp; i < n; i += 2 * NW) {
        const int i2 = i + NW < n ? i + NW : i;
        const double* r1 = X + i * ld;
        const double* r2 = X + i2 * ld;
        double s1 = 0.0, s2 = 0.0;
        for (int j = lane; j < n; j += 32) {
          const double qj = q[j];
          s1 = fma(r1[j], qj, s1);
          s2 = fma(r2[j], qj, s2);
        }
        s1 = warp_sum(s1);
        s2 = warp_sum(s2);
        const double w1 = s1 - beta * qp[i];
        qw = fma(q[i], w1, qw);
        ww = fma(w1, w1, ww);
        if (lane == 0) w[i] = w1;
        if (i2 != i) {
          const double w2 = s2 - beta * qp[i2];
          qw = fma(q[i2], w2, qw);
          ww = fma(w2, w2, ww);
          if (lane == 0) w[i2] = w2;
        }
      }
      double* part = red + 32 * (k & 1);
      if (lane == 0) { part[warp] = qw; part[16 + warp] = ww; }
      __syncthreads();
      qw = 0.0;
      ww = 0.0;
#pragma unroll
      for (int t = 0; t < NW; ++t) { qw += part[t]; ww += part[16 + t]; }
      const double alpha = qw, nb = sqrt(fmax(ww - alpha * alpha, 0.0));
      al[k] = alpha;
      be[k] = nb;
      if (!(nb > 1e-10 * (fabs(alpha) + 1.0))) { broke = true; break; }
      const double rnb = 1.0 / nb;
      for (int i = threadIdx.x; i < n; i += NT) {
        const double qi = q[i];
        qp[i] = qi;
        q[i] = (w[i] - alpha * qi) * rnb;
      }
      beta = nb;
      __syncthreads();
    }
    if (!broke) {
      double llo, lhi;
      lanczos_bounds<kLanczosSteps>(al, be, be[kLanczosSteps - 1], llo, lhi);
      if (llo == llo && lhi == lhi) {
        lo = fmax(lo, llo);
        hi = fmin(hi, lhi);
      }
    }
  }
  if (!(hi - lo > 1e-12)) hi = lo + 1.0;  // F a multiple of I (or not finite: caught later)
  const double inv = 1.0 / (hi - lo);
  double s1 = 0.0, s2 = 0.0;
  for (int t = threadIdx.x; t < n * n; t += NT) {
    const int r = t / n, c = t - r * n;
    const double v = ((r == c ? hi : 0.0) - X[r * ld + c]) * inv;
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
    rowI[u] = (I * 16 + g) * ld + 2 * q;
    rowJ[u] = (J * 16 + g) * ld + 2 * q;
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[u][k][0] = acc[u][k][1] = 0.0;
  }
  // Lane (g, q) loads columns k0 + 2q, k0 + 2q + 1 of its rows as one 16-byte load; the first
  // DMMA takes the even columns, the second the odd ones (the same permutation of k for A and
  // B, so the sum is unchanged).  Row stride ld = n16 + 8 keeps a quarter-warp's two rows in
  // opposite halves of the banks.
  for (int k0 = 0; k0 < n16; k0 += 8) {
#pragma unroll
    for (int u = 0; u < MAXST; ++u) {
      if (warp + u * NW < cnt) {
        const double2 a0 = *reinterpret_cast<const double2*>(X + rowI[u] + k0);
        const double2 a1 = *reinterpret_cast<const double2*>(X + rowI[u] + 8 * ld + k0);
        const double2 b0 = *reinterpret_cast<const double2*>(X + rowJ[u] + k0);
        const double2 b1 = *reinterpret_cast<const double2*>(X + rowJ[u] + 8 * ld + k0);
        const bool off = rowI[u] != rowJ[u];
        dmma884(acc[u][0][0], acc[u][0][1], a0.x, b0.x);
        if (off) dmma884(acc[u][1][0], acc[u][1][1], a0.x, b1.x);
        dmma884(acc[u][2][0], acc[u][2][1], a1.x, b0.x);
        dmma884(acc[u][3][0], acc[u][3][1], a1.x, b1.x);
        dmma884(acc[u][0][0], acc[u][0][1], a0.y, b0.y);
        if (off) dmma884(acc[u][1][0], acc[u][1][1], a0.y, b1.y);
        dmma884(acc[u][2][0], acc[u][2][1], a1.y, b0.y);
        dmma884(acc[u][3][0], acc[u][3][1], a1.y, b1.y);
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
// number of products, or -1 (no convergence, wrong trace or a non-finite value).  lz: 3 n
// doubles of shared scratch; red: 64 doubles.
// The recursion from the current X (trace t1, squared norm t2) on, products numbered from it0.
template <int NT>
__device__ int purify_fp64_loop(double* X, int n16, int ld, int nocc, double* red, double t1,
                                double t2, int it0, bool mixed_finish = false) {
  int tail = -1;
  for (int it = it0; it <= kPurifyMaxIter; ++it) {
    if (!(fabs(t1) < INFINITY) || !(fabs(t2) < INFINITY)) return -1;
    if (mixed_finish) {  // the mixed form: done at kMixedIdemFinal, no tail
      if (fabs(t1 - t2) < kMixedIdemFinal) tail = 0;
    } else {
      if (tail < 0 && fabs(t1 - t2) < kPurifyIdem) tail = kPurifyTail;
      if (fabs(t1 - t2) < kPurifyIdemFinal) tail = 0;
    }
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

template <int NT>
__device__ int block_purify(const double* F, int n, int nocc, double* X, double* lz,
                            double* red) {
  const int ld = purify_ld(n), n16 = purify_n16(n);
  double t1, t2;
  purify_init<NT>(F, n, X, ld, lz, red, t1, t2);
  return purify_fp64_loop<NT>(X, n16, ld, nocc, red, t1, t2, 0);
}

// ------------------------------------------------------------------------------------------
// Mixed precision on the 5th-generation tensor cores (SOLVER_PURIFY_MIXED, 64 < n16 <= 128;
// larger orders up to 160 go on to block_purify_mixed_wide below):
// the products of the recursion run as tcgen05.mma kind::tf32 with the accumulator in tensor
// memory, X split into two TF32 parts (hi = X with the low 13 mantissa bits cleared, lo = X - hi)
// and X^2 ~ hi hi + hi lo + lo hi (FP32-level accuracy, "3xTF32").  hi and lo sit in shared
// memory in the K-major no-swizzle canonical layout of the MMA (8-row x 16-byte core matrices:
// element (r, k) at float ((r/8)(n16/4) + k/4) 32 + (r%8) 4 + k%4, 128 rows, rows past n16
// zero), so one descriptor pair serves as A (M = 128) and, X being symmetric, as B (N = n16).
// One thread issues the 3 n16 / 8 MMAs of a product and commits them to an mbarrier; every warp
// then reads its 32 rows x 32 columns of X^2 from tensor memory (tcgen05.ld 32x32b), forms the
// branch, re-splits and writes back.  When tr(X - X^2) < kPurifyTensorSwitch, X is symmetrised
// into FP64 and the recursion finishes with FP64 products (purify_fp64_loop), so the result has
// FP64 idempotency and the FP32 phase perturbs the occupied subspace only at the 1e-6 level.

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ int kmajor_index(int r, int k, int K) {
  return ((r >> 3) * (K >> 2) + (k >> 2)) * 32 + (r & 7) * 4 + (k & 3);
}
// Shared-memory matrix descriptor: start address, leading (K-direction) and stride
// (8-row-group) byte offsets, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}
// Instruction descriptor: FP32 accumulator, TF32 A and B, both K-major, M x N.
__device__ __forceinline__ uint32_t umma_idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Bounded wait for the MMAs of one product (x >= 64 ns sleep: a few hundred ms at most).  The
// first wait of a product takes its bound from the caller (the context's wait limit, this value
// by default); after a timed-out wait the second, recovery wait always uses this bound, so the
// tensor memory is given back only after the MMAs that write it have completed.
constexpr long long kMbarSpins = 1 << 22;
// FP32 products until tr(X - X^2) falls below this (3xTF32 keeps X to ~1e-7, so the
// idempotency error is still well above its FP32 floor of ~1e-5 here)
constexpr double kPurifyTensorSwitch = 1e-4;

// Splits v into its TF32 head and the FP32 remainder at canonical position idx.
__device__ __forceinline__ void put_split(float* hi, float* lo, int idx, float v) {
  const float h = __uint_as_float(__float_as_uint(v) & 0xFFFFE000u);
  hi[idx] = h;
  lo[idx] = v - h;
}

// Reads 16 consecutive accumulator columns of the warp's 32 tensor-memory lanes (one row per
// thread); 16 at a time keeps the epilogue within the 128 registers a 512-thread CTA allows.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;");
}

template <int NT>
__device__ __noinline__ int block_purify_mixed_wide(const double* F, int n, int nocc, double* X,
                                                    double* lz, double* red, long long spins);

template <int NT>
__device__ __noinline__ int block_purify_mixed(const double* F, int n, int nocc, double* X,
                                               double* lz, double* red, long long spins) {
  constexpr int NW = NT / 32;
  static_assert(NT == 512, "the tensor-memory epilogue maps 16 warps onto 4 x 4 tiles of 32");
  if (purify_n16(n) > 128) return block_purify_mixed_wide<NT>(F, n, nocc, X, lz, red, spins);
  const int ld = purify_ld(n), n16 = purify_n16(n);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double t1, t2;
  purify_init<NT>(F, n, X, ld, lz, red, t1, t2);
  // ---- X (FP64, row stride ld) -> hi / lo (FP32 canonical, 128 rows) through registers ----
  float* hi = reinterpret_cast<float*>(X);
  float* lo = hi + 128 * n16;
  constexpr int kPer = 128 * 128 / NT;  // elements per thread (n16 <= 128)
  float keep[kPer];
#pragma unroll
  for (int e = 0; e < kPer; ++e) {
    const int t = threadIdx.x + e * NT, r = t / 128, c = t % 128;
    keep[e] = (r < n16 && c < n16) ? (float)X[r * ld + c] : 0.0f;
  }
  __syncthreads();
#pragma unroll
  for (int e = 0; e < kPer; ++e) {
    const int t = threadIdx.x + e * NT, r = t / 128, c = t % 128;
    if (c < n16) put_split(hi, lo, kmajor_index(r, c, n16), keep[e]);
  }
  uint64_t* mbar = reinterpret_cast<uint64_t*>(lz);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(lz + 1);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  if (warp == 0)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(128));
  asm volatile("fence.proxy.async.shared::cta;");
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tslot;
  const uint32_t idesc = umma_idesc_tf32(128, n16);
  const uint32_t lbo = 128, sbo = (uint32_t)(n16 / 4) * 128;
  const int row = 32 * (warp & 3) + lane, c0 = (warp >> 2) * 32;
  const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)c0;
  // the 32 elements (row, c0 .. c0 + 31) this thread rewrites after every product stay in
  // registers, so the epilogue reads only tensor memory
  float xr[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    const int c = c0 + j;
    xr[j] = 0.0f;
    if (row < n16 && c < n16) {
      const int idx = kmajor_index(row, c, n16);
      xr[j] = hi[idx] + lo[idx];
    }
  }
  int it = 0, status = 0;
  uint32_t phase = 0;
  for (; it < kPurifyMaxIter; ++it) {
    if (!(fabs(t1) < INFINITY) || !(fabs(t2) < INFINITY)) { status = -1; break; }
    if (fabs(t1 - t2) < kPurifyTensorSwitch) break;
    const double n_o = (double)nocc;
    const bool sq = fabs(t2 - n_o) < fabs(2.0 * t1 - t2 - n_o);
    if (threadIdx.x == 0) {
      int first = 1;
      for (int k0 = 0; k0 < n16; k0 += 8) {
        const uint32_t off = (uint32_t)(k0 / 4) * 128;
        const uint64_t dh = umma_smem_desc(smem_u32(hi) + off, lbo, sbo);
        const uint64_t dl = umma_smem_desc(smem_u32(lo) + off, lbo, sbo);
        const uint64_t da[3] = {dh, dh, dl}, db[3] = {dh, dl, dh};
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                       "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                       "l"(da[q]), "l"(db[q]), "r"(idesc), "r"(first ? 0 : 1));
          first = 0;
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(mbar)));
    }
    uint32_t done = 0;
    for (long long spin = 0; spin < spins && !done; ++spin) {
      asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                   "selp.u32 %0, 1, 0, p;\n\t}"
                   : "=r"(done)
                   : "r"(smem_u32(mbar)), "r"(phase));
      if (!done) __nanosleep(64);
    }
    // every thread takes the same branch: the MMAs completed for all or the step is abandoned
    if (__syncthreads_or(!done)) {
      status = -2;
      break;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;");
    double s1 = 0.0, s2 = 0.0;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      uint32_t v[16];
      tmem_ld16(taddr + (uint32_t)(16 * half), v);
#pragma unroll
      for (int g = 0; g < 4; ++g) {  // four columns = 16 contiguous bytes of a core matrix row
        const int c = c0 + 16 * half + 4 * g;
        if (row < n16 && c < n16) {
          float h4[4], l4[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int j = 16 * half + 4 * g + q;
            const float d = __uint_as_float(v[4 * g + q]);
            const float nv = sq ? d : fmaf(2.0f, xr[j], -d);
            xr[j] = nv;
            h4[q] = __uint_as_float(__float_as_uint(nv) & 0xFFFFE000u);
            l4[q] = nv - h4[q];
            if (row == c + q) s1 += nv;
            s2 = fma((double)nv, (double)nv, s2);
          }
          const int idx = kmajor_index(row, c, n16);
          *reinterpret_cast<float4*>(hi + idx) = make_float4(h4[0], h4[1], h4[2], h4[3]);
          *reinterpret_cast<float4*>(lo + idx) = make_float4(l4[0], l4[1], l4[2], l4[3]);
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    double* part = red + 32 * (it & 1);
    if (lane == 0) { part[warp] = s1; part[16 + warp] = s2; }
    asm volatile("fence.proxy.async.shared::cta;");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();  // X rewritten, tensor memory read: the next product may start
    asm volatile("tcgen05.fence::after_thread_sync;");
    s1 = 0.0;
    s2 = 0.0;
#pragma unroll
    for (int k = 0; k < NW; ++k) { s1 += part[k]; s2 += part[16 + k]; }
    t1 = s1;
    t2 = s2;
  }
  if (status == -2) {
    // MMAs still outstanding after the bounded wait: wait once more (bounded) before giving the
    // tensor memory back; the step is then diagonalised instead
    uint32_t done = 0;
    for (int spin = 0; spin < kMbarSpins && !done; ++spin) {
      asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                   "selp.u32 %0, 1, 0, p;\n\t}"
                   : "=r"(done)
                   : "r"(smem_u32(mbar)), "r"(phase));
      if (!done) __nanosleep(64);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
  if (threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(mbar)));
  if (status < 0) return -1;
  if (it == kPurifyMaxIter) return -1;
  // ---- back to FP64, symmetrised (the tensor-core products are not bit-symmetric) ----
  double back[kPer];
#pragma unroll
  for (int e = 0; e < kPer; ++e) {
    const int t = threadIdx.x + e * NT, r = t / 128, c = t % 128;
    back[e] = 0.0;
    if (r < n16 && c < n16) {
      const int a = kmajor_index(r, c, n16), b = kmajor_index(c, r, n16);
      back[e] = 0.5 * (((double)hi[a] + (double)lo[a]) + ((double)hi[b] + (double)lo[b]));
    }
  }
  __syncthreads();
  double s1 = 0.0, s2 = 0.0;
#pragma unroll
  for (int e = 0; e < kPer; ++e) {
    const int t = threadIdx.x + e * NT, r = t / 128, c = t % 128;
    if (r < n16 && c < n16) {
      X[r * ld + c] = back[e];
      if (r == c) s1 += back[e];
      s2 = fma(back[e], back[e], s2);
    }
  }
  for (int t = threadIdx.x; t < n16 * 4; t += NT) X[(t >> 2) * ld + n16 + (t & 3)] = 0.0;  // pad
  block_sum2<NT>(s1, s2, red);
  return purify_fp64_loop<NT>(X, n16, ld, nocc, red, s1, s2, it, true);
}

// ------------------------------------------------------------------------------------------
// The same mixed form for n16 = 144 and 160 (nao 129-160), where X is taller than one M = 128
// tile.  hi / lo hold all n16 rows (2 x n16 x n16 floats inside X's region).  A product is two
// accumulators: D1 = X[0:128, :] X (M = 128, N = n16, tensor-memory columns 0 .. n16-1) and
// D2 = X[n16-128 : n16, :] X[:, 128 : n16] (M = 128, N = n16 - 128, columns kWideCorner ..),
// whose last n16 - 128 rows are the corner X^2[128:n16, 128:n16].  The block
// X^2[128:n16, 0:128] is the transpose of D1's columns 128 .. n16-1 (X^2 is symmetric), so the
// warps that read those columns write each new element twice, at (r, c) and (c, r).  Tasks of
// 32 rows x 32 columns: every warp one tile of D1[0:128, 0:128]; warps 0-3 also D1's fifth
// column tile; warp 7 the corner from D2.  The old X of an element is read back from hi + lo.

constexpr int kWideCorner = 192;  // tensor-memory column of D2 (256 columns allocated)

// Row and column of the t-th element of a lower triangle stored row by row.
__device__ __forceinline__ void tri_rc(int t, int& r, int& c) {
  r = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
  while (r * (r + 1) / 2 > t) --r;
  while ((r + 1) * (r + 2) / 2 <= t) ++r;
  c = t - r * (r + 1) / 2;
}

// Half of a 32-column task of the wide epilogue: row `row` of X, columns cb .. cb + 15 (those
// < n16), X^2 values in v.  Writes the new X into hi / lo at (row, c) and, with `mirror`, at (c, row);
// adds to the trace and squared-norm sums (a mirrored element counts twice in the norm).
__device__ __forceinline__ void wide_update(float* hi, float* lo, int n16, int row, int cb,
                                            const uint32_t (&v)[16], bool sq, bool mirror,
                                            double& s1, double& s2) {
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    const int c = cb + 4 * g;
    if (c < n16) {
      const int idx = kmajor_index(row, c, n16);
      const float4 oh = *reinterpret_cast<const float4*>(hi + idx);
      const float4 ol = *reinterpret_cast<const float4*>(lo + idx);
      const float old[4] = {oh.x + ol.x, oh.y + ol.y, oh.z + ol.z, oh.w + ol.w};
      float h4[4], l4[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float d = __uint_as_float(v[4 * g + q]);
        const float nv = sq ? d : fmaf(2.0f, old[q], -d);
        h4[q] = __uint_as_float(__float_as_uint(nv) & 0xFFFFE000u);
        l4[q] = nv - h4[q];
        if (row == c + q) s1 += nv;
        s2 = fma(mirror ? 2.0 * (double)nv : (double)nv, (double)nv, s2);
        if (mirror) {
          const int tdx = kmajor_index(c + q, row, n16);
          hi[tdx] = h4[q];
          lo[tdx] = l4[q];
        }
      }
      *reinterpret_cast<float4*>(hi + idx) = make_float4(h4[0], h4[1], h4[2], h4[3]);
      *reinterpret_cast<float4*>(lo + idx) = make_float4(l4[0], l4[1], l4[2], l4[3]);
    }
  }
}

template <int NT>
__device__ __noinline__ int block_purify_mixed_wide(const double* F, int n, int nocc, double* X,
                                                    double* lz, double* red, long long spins) {
  constexpr int NW = NT / 32;
  static_assert(NT == 512, "the tensor-memory epilogue maps 16 warps onto 4 x 4 tiles of 32");
  const int ld = purify_ld(n), n16 = purify_n16(n), R = n16 - 128;  // R = 16 or 32
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double t1, t2;
  purify_init<NT>(F, n, X, ld, lz, red, t1, t2);
  // ---- X (FP64, lower triangle, row stride ld) -> hi / lo (both triangles) ----
  float* hi = reinterpret_cast<float*>(X);
  float* lo = hi + n16 * n16;
  constexpr int kTri = (160 * 161 / 2 + NT - 1) / NT;
  const int ntri = n16 * (n16 + 1) / 2;
  float keep[kTri];
#pragma unroll
  for (int e = 0; e < kTri; ++e) {
    const int t = threadIdx.x + e * NT;
    keep[e] = 0.0f;
    if (t < ntri) {
      int r, c;
      tri_rc(t, r, c);
      keep[e] = (float)X[r * ld + c];
    }
  }
  __syncthreads();
#pragma unroll
  for (int e = 0; e < kTri; ++e) {
    const int t = threadIdx.x + e * NT;
    if (t < ntri) {
      int r, c;
      tri_rc(t, r, c);
      put_split(hi, lo, kmajor_index(r, c, n16), keep[e]);
      if (r != c) put_split(hi, lo, kmajor_index(c, r, n16), keep[e]);
    }
  }
  uint64_t* mbar = reinterpret_cast<uint64_t*>(lz);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(lz + 1);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  if (warp == 0)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(256));
  asm volatile("fence.proxy.async.shared::cta;");
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tslot;
  const uint32_t id1 = umma_idesc_tf32(128, n16), id2 = umma_idesc_tf32(128, R);
  const uint32_t lbo = 128, sbo = (uint32_t)(n16 / 4) * 128;
  const uint32_t a2 = (uint32_t)(R / 8) * sbo, b2 = 16u * sbo;  // D2's first rows of A and B
  const int quad = warp & 3, row = 32 * quad + lane, c0 = (warp >> 2) * 32;
  const uint32_t tlane = (uint32_t)(32 * quad) << 16;
  int it = 0, status = 0;
  uint32_t phase = 0;
  for (; it < kPurifyMaxIter; ++it) {
    if (!(fabs(t1) < INFINITY) || !(fabs(t2) < INFINITY)) { status = -1; break; }
    if (fabs(t1 - t2) < kPurifyTensorSwitch) break;
    const double n_o = (double)nocc;
    const bool sq = fabs(t2 - n_o) < fabs(2.0 * t1 - t2 - n_o);
    if (threadIdx.x == 0) {
      const uint32_t h0 = smem_u32(hi), l0 = smem_u32(lo);
      for (int acc = 0; acc < 2; ++acc) {
        const uint32_t ao = acc ? a2 : 0u, bo = acc ? b2 : 0u, id = acc ? id2 : id1;
        const uint32_t d = tmem + (acc ? (uint32_t)kWideCorner : 0u);
        int first = 1;
        for (int k0 = 0; k0 < n16; k0 += 8) {
          const uint32_t off = (uint32_t)(k0 / 4) * 128;
          const uint64_t ah = umma_smem_desc(h0 + ao + off, lbo, sbo);
          const uint64_t al = umma_smem_desc(l0 + ao + off, lbo, sbo);
          const uint64_t bh = umma_smem_desc(h0 + bo + off, lbo, sbo);
          const uint64_t bl = umma_smem_desc(l0 + bo + off, lbo, sbo);
          const uint64_t da[3] = {ah, ah, al}, db[3] = {bh, bl, bh};
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                         "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
                         "l"(da[q]), "l"(db[q]), "r"(id), "r"(first ? 0 : 1));
            first = 0;
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(mbar)));
    }
    uint32_t done = 0;
    for (long long spin = 0; spin < spins && !done; ++spin) {
      asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                   "selp.u32 %0, 1, 0, p;\n\t}"
                   : "=r"(done)
                   : "r"(smem_u32(mbar)), "r"(phase));
      if (!done) __nanosleep(64);
    }
    if (__syncthreads_or(!done)) {
      status = -2;
      break;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;");
    double s1 = 0.0, s2 = 0.0;
    const int xr = n16 - 32 + lane;  // warp 7 (quadrant 3 of D2): lane l is row n16 - 32 + l
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const uint32_t h16 = (uint32_t)(16 * half);
      uint32_t v[16];
      tmem_ld16(tmem + tlane + (uint32_t)c0 + h16, v);
      wide_update(hi, lo, n16, row, c0 + 16 * half, v, sq, false, s1, s2);
      if (warp < 4) {  // D1's columns 128 .. n16-1: rows < 128 here, rows >= 128 by symmetry
        tmem_ld16(tmem + tlane + 128u + h16, v);
        wide_update(hi, lo, n16, row, 128 + 16 * half, v, sq, true, s1, s2);
      }
      if (warp == 7) {
        tmem_ld16(tmem + tlane + (uint32_t)kWideCorner + h16, v);
        if (xr >= 128) wide_update(hi, lo, n16, xr, 128 + 16 * half, v, sq, false, s1, s2);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    double* part = red + 32 * (it & 1);
    if (lane == 0) { part[warp] = s1; part[16 + warp] = s2; }
    asm volatile("fence.proxy.async.shared::cta;");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();  // X rewritten, tensor memory read: the next product may start
    asm volatile("tcgen05.fence::after_thread_sync;");
    s1 = 0.0;
    s2 = 0.0;
#pragma unroll
    for (int k = 0; k < NW; ++k) { s1 += part[k]; s2 += part[16 + k]; }
    t1 = s1;
    t2 = s2;
  }
  if (status == -2) {
    uint32_t done = 0;
    for (int spin = 0; spin < kMbarSpins && !done; ++spin) {
      asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                   "selp.u32 %0, 1, 0, p;\n\t}"
                   : "=r"(done)
                   : "r"(smem_u32(mbar)), "r"(phase));
      if (!done) __nanosleep(64);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256));
  if (threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(mbar)));
  if (status < 0) return -1;
  if (it == kPurifyMaxIter) return -1;
  // ---- back to FP64 (lower triangle averaged with the upper, written to both) ----
  double back[kTri];
#pragma unroll
  for (int e = 0; e < kTri; ++e) {
    const int t = threadIdx.x + e * NT;
    back[e] = 0.0;
    if (t < ntri) {
      int r, c;
      tri_rc(t, r, c);
      const int a = kmajor_index(r, c, n16), b = kmajor_index(c, r, n16);
      back[e] = 0.5 * (((double)hi[a] + (double)lo[a]) + ((double)hi[b] + (double)lo[b]));
    }
  }
  __syncthreads();
  double s1 = 0.0, s2 = 0.0;
#pragma unroll
  for (int e = 0; e < kTri; ++e) {
    const int t = threadIdx.x + e * NT;
    if (t < ntri) {
      int r, c;
      tri_rc(t, r, c);
      X[r * ld + c] = back[e];
      X[c * ld + r] = back[e];
      if (r == c) s1 += back[e];
      s2 = fma(r == c ? back[e] : 2.0 * back[e], back[e], s2);
    }
  }
  for (int t = threadIdx.x; t < n16 * 4; t += NT) X[(t >> 2) * ld + n16 + (t & 3)] = 0.0;  // pad
  block_sum2<NT>(s1, s2, red);
  return purify_fp64_loop<NT>(X, n16, ld, nocc, red, s1, s2, it, true);
}

// Above nao 160 X does not fit in shared memory: X and Y (n16 x n16, row stride n16 + 8) live
// in global memory (L1/L2-resident panels).  A warp takes one super-tile at a time, keeps its
// four 8 x 8 accumulators in registers and writes the new values straight into Y, reading the
// old X for the 2X - X^2 branch; the caller swaps X and Y after each step.
template <int NT>
__device__ __noinline__ void purify_step_global(const double* __restrict__ X,
                                                double* __restrict__ Y, int n16, int ld, bool sq,
                                                double* red, int buf, double& t1, double& t2) {
  constexpr int NW = NT / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, q = lane & 3;
  const int nst = n16 >> 4, cnt = nst * (nst + 1) / 2;
  double s1 = 0.0, s2 = 0.0;
  int I = 0, J = 0;
  if (warp < cnt) tri_inverse(warp, I, J);
  for (int st = warp; st < cnt; st += NW) {
    const int64_t ri = (int64_t)(I * 16 + g) * ld + q, rj = (int64_t)(J * 16 + g) * ld + q;
    double acc[4][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    const bool diag = I == J;
    for (int k0 = 0; k0 < n16; k0 += 4) {
      const double a0 = X[ri + k0], a1 = X[ri + 8 * ld + k0];
      const double b0 = X[rj + k0], b1 = X[rj + 8 * ld + k0];
      dmma884(acc[0][0], acc[0][1], a0, b0);
      if (!diag) dmma884(acc[1][0], acc[1][1], a0, b1);
      dmma884(acc[2][0], acc[2][1], a1, b0);
      dmma884(acc[3][0], acc[3][1], a1, b1);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int r = I * 16 + (k >> 1) * 8 + g;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int c = J * 16 + (k & 1) * 8 + 2 * q + e;
        if (r >= c) {
          const double x2 = acc[k][e];
          const double v = sq ? x2 : fma(2.0, X[(int64_t)r * ld + c], -x2);
          Y[(int64_t)r * ld + c] = v;
          if (r != c) Y[(int64_t)c * ld + r] = v;
          if (r == c) s1 += v;
          s2 = fma(r == c ? v : 2.0 * v, v, s2);
        }
      }
    }
    // next super-tile of this warp: advance the packed index by NW
    J += NW;
    while (J > I) { J -= I + 1; ++I; }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  double* part = red + 32 * buf;
  if (lane == 0) { part[warp] = s1; part[16 + warp] = s2; }
  __syncthreads();  // Y and the partial sums complete
  s1 = 0.0;
  s2 = 0.0;
#pragma unroll
  for (int k = 0; k < NW; ++k) { s1 += part[k]; s2 += part[16 + k]; }
  t1 = s1;
  t2 = s2;
}

// block_purify with X and its partner Y in global memory (nao > 160).  Returns the number of
// products and leaves the result in *Xout (X or Y), or -1.
template <int NT>
__device__ int block_purify_global(const double* F, int n, int nocc, double* X, double* Y,
                                   double* lz, double* red, double** Xout) {
  const int ld = purify_ld(n), n16 = purify_n16(n);
  double t1, t2;
  purify_init<NT>(F, n, X, ld, lz, red, t1, t2);
  // Y's padding must be zero as X's is: the steps only write the n16 x n16 block
  for (int64_t t = threadIdx.x; t < (int64_t)n16 * ld; t += NT) Y[t] = 0.0;
  __syncthreads();
  int tail = -1;
  for (int it = 0; it <= kPurifyMaxIter; ++it) {
    if (!(fabs(t1) < INFINITY) || !(fabs(t2) < INFINITY)) return -1;
    if (tail < 0 && fabs(t1 - t2) < kPurifyIdem) tail = kPurifyTail;
    if (fabs(t1 - t2) < kPurifyIdemFinal) tail = 0;
    if (tail == 0) {
      *Xout = X;
      return fabs(t1 - (double)nocc) < kPurifyTraceTol ? it : -1;
    }
    if (tail > 0) --tail;
    if (it == kPurifyMaxIter) break;
    const double n_o = (double)nocc;
    const bool sq = fabs(t2 - n_o) < fabs(2.0 * t1 - t2 - n_o);
    purify_step_global<NT>(X, Y, n16, ld, sq, red, it & 1, t1, t2);
    double* tmp = X;
    X = Y;
    Y = tmp;
  }
  return -1;
}

// P (packed lower triangle) = 2 X, or with density damping d > 0
// P = (1 - d) 2 X + d P_previous (P holds the previous step's density on entry).
__device__ inline void purify_density(const double* X, int n, double* P, double d) {
  const int ld = purify_ld(n);
  const int64_t np = tri(n);
  for (int64_t t = threadIdx.x; t < np; t += blockDim.x) {
    int i, j;
    tri_inverse(t, i, j);
    const double p = 2.0 * X[(int64_t)i * ld + j];
    P[t] = d > 0.0 ? fma(d, P[t] - p, p) : p;
  }
}

}  // namespace sgb
