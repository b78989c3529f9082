// Purification of one large molecule on the whole GPU, as ONE persistent cooperative launch per
// SCF step: every product X^2 of the trace-correcting recursion (purify.cuh), the branch
// X <- X^2 or 2X - X^2, the trace and squared-norm sums that choose the next branch, and the
// convergence test all run on the device; products are separated by a grid barrier, so there
// is no host round trip between them.  This replaces the host-driven loop of library DSYRK
// calls; the density it produces is the same projector (the aufbau density of the reference's
// dsyev eigenvectors, densitymatrix.cpp:40-56).
//
// Layout: X and its partner Y are np x np row-major (np = nao rounded up to the tile, zero
// padding, which stays zero), symmetric, both triangles stored.  A product is computed tile by
// tile over the lower triangle of BM x BM tiles, dealt round-robin to the CTAs (a fixed
// assignment, so every sum has a fixed order).
//
// Per tile: the row panels X[I-tile, :] and X[J-tile, :] (X^2 = X X^T for symmetric X) stream
// through shared memory in k-blocks of 16 doubles, loaded by TMA (one 128-byte swizzled row per
// panel row; the swizzle spreads a warp's 16-byte fragment loads over all banks) into a ring of
// stages guarded by full / empty mbarriers: thread 0 issues the loads a ring ahead,
// every warp runs FP64 tensor-core MMAs (DMMA m8n8k4) on register accumulators, then writes
// the new X into Y (the element and its mirror) and adds to the trace / norm sums.  The panels
// are L2-resident up to a few thousand AOs; above, each k-block is read by nt CTAs from HBM.
//
// Every wait is bounded (the context's wait limit): a timed-out mbarrier wait or grid barrier
// sets the error flag, every CTA leaves at its next barrier, thread 0 first waits (bounded) for
// the loads it issued that are still in flight, and the host reports the failure.
#pragma once
#include "dmma_tiles.cuh"
#include "grid_scf.cuh"

namespace sgb {

struct GridPurifyArgs {
  int np;            // padded order: row stride of both buffers, a multiple of the tile
  int nocc;
  double* buf[2];    // X_0 in buf[0]
  double* partial;   // 2 (product parity) x 2 (sums) x gridDim
  const double* t0;  // tr X_0, ||X_0||^2
  int* result;       // [0] products (>= 0), -1 (no convergence / wrong trace / non-finite),
                     // -2 (a wait gave up); [1] index of the buffer holding the final X
  GridBarrier bar;
  long long spins;   // polls of each mbarrier wait
  int it0;           // products already done (the mixed form's FP32 phase)
  int mixed_finish;  // the mixed form: done at kMixedIdemFinal, no tail
};

template <class C>
__global__ void __launch_bounds__(C::THREADS, 1)
    k_grid_purify(const __grid_constant__ CUtensorMap map0,
                  const __grid_constant__ CUtensorMap map1, GridPurifyArgs a) {
  extern __shared__ unsigned char smem_raw[];
  GpRing ring;
  ring.tiles = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                ~uintptr_t(1023));
  ring.full = reinterpret_cast<uint64_t*>(ring.tiles + C::STAGES * C::STAGE_BYTES);
  ring.empty = ring.full + C::STAGES;
  __shared__ double red[2][C::WARPS + 1];
  __shared__ volatile int s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < C::STAGES; ++s) {
      mbar_init(ring.full + s, 1);
      mbar_init(ring.empty + s, C::WARPS);
    }
    mbar_fence_init();
    s_abort = 0;
    tma_prefetch_map(&map0);
    tma_prefetch_map(&map1);
  }
  __syncthreads();
  // ring steps per tile: np / (16 KB) rounded up; k-blocks past np read as zeros (TMA fills a
  // box's out-of-range part), so they add nothing to the products
  const int np = a.np, nt = np / C::BM, T = nt * (nt + 1) / 2;
  const int kblocks = (np + kGpK * C::KB - 1) / (kGpK * C::KB);
  const int G = gridDim.x;
  const int my_tiles = (int)blockIdx.x < T ? (T - 1 - (int)blockIdx.x) / G + 1 : 0;
  double* const buf0 = a.buf[0];
  double* const buf1 = a.buf[1];
  double t1 = a.t0[0], t2 = a.t0[1];
  int tail = -1, result = -1, cur = 0;
  for (int it = a.it0;; ++it) {
    // ---- the decision of purify_fp64_loop, identical in every thread of every CTA ----
    if (!(fabs(t1) < INFINITY) || !(fabs(t2) < INFINITY)) { result = -1; break; }
    if (a.mixed_finish) {
      if (fabs(t1 - t2) < kMixedIdemFinal) tail = 0;
    } else {
      if (tail < 0 && fabs(t1 - t2) < kPurifyIdem) tail = kPurifyTail;
      if (fabs(t1 - t2) < kPurifyIdemFinal) tail = 0;
    }
    if (tail == 0) {
      result = fabs(t1 - (double)a.nocc) < kPurifyTraceTol ? it : -1;
      break;
    }
    if (tail > 0) --tail;
    if (it == kPurifyMaxIter) { result = -1; break; }
    const double n_o = (double)a.nocc;
    const bool sq = fabs(t2 - n_o) < fabs(2.0 * t1 - t2 - n_o);
    const CUtensorMap* map = cur ? &map1 : &map0;
    const double* X = cur ? buf1 : buf0;  // selects, not an indexed parameter array (which
    double* Y = cur ? buf0 : buf1;        // would be copied to local memory)
    double s1 = 0.0, s2 = 0.0;
    gp_product<C>(ring, map, X, Y, np, np, kblocks, blockIdx.x, G, my_tiles, sq, a.spins, &s_abort,
                  a.bar.err, s1, s2);
    // ---- this CTA's sums, then every CTA's in a fixed order ----
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
      red[0][warp] = s1;
      red[1][warp] = s2;
    }
    __syncthreads();
    double* part = a.partial + (it & 1) * 2 * G;
    if (threadIdx.x == 0) {
      double b1 = 0.0, b2 = 0.0;
      for (int w = 0; w < C::WARPS; ++w) { b1 += red[0][w]; b2 += red[1][w]; }
      __stcg(part + blockIdx.x, b1);
      __stcg(part + G + blockIdx.x, b2);
    }
    fence_proxy_async_global();  // Y is read by TMA in the next product
    if (!grid_barrier(a.bar) || s_abort) { result = -2; break; }
    if (warp == 0) {
      double u1 = 0.0, u2 = 0.0;
      for (int i = lane; i < G; i += 32) {
        u1 += __ldcg(part + i);
        u2 += __ldcg(part + G + i);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        u1 += __shfl_xor_sync(0xffffffffu, u1, o);
        u2 += __shfl_xor_sync(0xffffffffu, u2, o);
      }
      if (lane == 0) { red[0][C::WARPS] = u1; red[1][C::WARPS] = u2; }
    }
    __syncthreads();
    t1 = red[0][C::WARPS];
    t2 = red[1][C::WARPS];
    cur ^= 1;
    __syncthreads();  // red is rewritten by the next product
  }
  if (threadIdx.x == 0 && result == -2) {
    // loads still in flight land in this CTA's shared memory: wait for them (bounded) before
    // the CTA can exit
    for (long long c = ring.consumed; c < ring.issued; ++c)
      mbar_wait(ring.full + (int)(c % C::STAGES), (uint32_t)((c / C::STAGES) & 1), kMbarSpins);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.result[0] = result;
    a.result[1] = cur;
  }
}

// X_0 = (hi I - F) / (hi - lo) into the padded np x np buffer (zero padding); block partials of
// tr X_0 and ||X_0||^2, finished in a fixed order into out[0..1] by the last block.
__global__ void k_gp_init(int n, int np, const double* __restrict__ F, const double* lohi,
                          double* X, double* partial, unsigned* count, double* out) {
  const double lo = lohi[0], hi = lohi[1], inv = 1.0 / (hi - lo);
  const int64_t nn = (int64_t)np * np;
  double s1 = 0.0, s2 = 0.0;
  for (int64_t t = gtid(); t < nn; t += gstride()) {
    const int64_t i = t / np, j = t - i * np;
    double v = 0.0;
    if (i < n && j < n) {
      v = ((i == j ? hi : 0.0) - F[i * n + j]) * inv;
      if (i == j) s1 += v;
      s2 = fma(v, v, s2);
    }
    X[t] = v;
  }
  finalize_sums2(s1, s2, partial, count, out);
}

// FP32 X (n x n, symmetric) of the mixed form's first phase, widened into the padded FP64
// buffer, with the sums of k_gp_init.
__global__ void k_gp_widen32(int n, int np, const float* __restrict__ X32, double* X,
                             double* partial, unsigned* count, double* out) {
  const int64_t nn = (int64_t)np * np;
  double s1 = 0.0, s2 = 0.0;
  for (int64_t t = gtid(); t < nn; t += gstride()) {
    const int64_t i = t / np, j = t - i * np;
    double v = 0.0;
    if (i < n && j < n) {
      v = (double)X32[i * n + j];
      if (i == j) s1 += v;
      s2 = fma(v, v, s2);
    }
    X[t] = v;
  }
  finalize_sums2(s1, s2, partial, count, out);
}

// P = 2 X (packed) from the padded buffer, mixed with the previous P by the damping factor d
// when d > 0.
__global__ void k_gp_density(int n, int np, const double* __restrict__ X, double* P, double d) {
  for (int64_t t = gtid(); t < tri(n); t += gstride()) {
    int i, j;
    tri_inverse(t, i, j);
    const double p = 2.0 * X[(int64_t)i * np + j];
    P[t] = d > 0.0 ? fma(d, P[t] - p, p) : p;
  }
}

// X (padded, symmetric) -> X in the n x n layout of the rest of the grid path (G), for the DIIS
// commutator that follows a purified density.
__global__ void k_gp_unpad(int n, int np, const double* __restrict__ X, double* out) {
  const int64_t nn = (int64_t)n * n;
  for (int64_t t = gtid(); t < nn; t += gstride()) {
    const int64_t i = t / n, j = t - i * n;
    out[t] = X[i * np + j];
  }
}

}  // namespace sgb
