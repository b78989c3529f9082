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
#include "grid_scf.cuh"
#include "purify.cuh"
#include "tma.cuh"

namespace sgb {

constexpr int kGpK = 16;  // doubles per k-block: one 128-byte swizzle row per panel row

// BM x BM tiles, WGM x WGN warps, KB k-blocks (TMA boxes per operand) per ring stage,
// STAGES stages.  A stage's k-blocks are consumed one after the other; more (and wider) stages
// keep more loads in flight, which the small tiles need: their MMAs per k-block take a few
// hundred cycles, far less than a load's latency.
template <int BM_, int WGM_, int WGN_, int KB_, int STAGES_>
struct GpCfg {
  static constexpr int BM = BM_, WGM = WGM_, WGN = WGN_, KB = KB_, STAGES = STAGES_;
  static constexpr int WM = BM / WGM, WN = BM / WGN;  // warp tile
  static constexpr int FM = WM / 8, FN = WN / 8;      // 8 x 8 DMMA fragments per warp tile
  static constexpr int WARPS = WGM * WGN;
  static constexpr int THREADS = WARPS * 32;
  static constexpr int BOX_BYTES = BM * 128;           // one operand's k-block
  static constexpr int STAGE_BYTES = 2 * KB * BOX_BYTES;
  static constexpr size_t SMEM = 1024 + (size_t)STAGES * STAGE_BYTES + 2 * STAGES * 8;
  static_assert(WM % 8 == 0 && WN % 8 == 0, "warp tiles are whole fragments");
  static_assert(BOX_BYTES % 1024 == 0, "the 128-byte swizzle repeats every 1024 bytes");
};
// Measured on C2000H2002 (10002 AOs, one FP64 SCF): the 128 x 128 tile with 8 warps of
// 64 x 32 (240 registers a thread) and 3 k-blocks per stage in 2 stages ran 10.9 s; 2 x 3
// stages 11.0 s, 16 warps of 32 x 32 with 6 one-block stages 11.4 s, 8 warps with 6 one-block
// stages 13-15 s: every stage costs a barrier wait and arrive per warp and a refill by thread 0,
// so wider stages win while two of them still cover a load's latency.
using GpLarge = GpCfg<128, 2, 4, 3, 2>;     // 8 warps of 64 x 32, 2 x 96 KB stages
using GpMid = GpCfg<64, 2, 4, 2, 6>;        // 8 warps of 32 x 16, 6 x 32 KB stages
using GpSmall = GpCfg<32, 2, 2, 4, 3>;      // 4 warps of 16 x 16, 3 x 32 KB stages (2 CTAs/SM)
// alternatives of the 128 x 128 tile, selectable with SGB_GRID_VARIANT=1 / 2 for sweeps
using GpLargeAlt1 = GpCfg<128, 2, 4, 2, 3>;  // 8 warps of 64 x 32, 3 x 64 KB stages
using GpLargeAlt2 = GpCfg<128, 4, 4, 1, 6>;  // 16 warps of 32 x 32, 6 x 32 KB stages

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
};

// The load ring.  Thread 0 issues the loads of ring steps STAGES ahead of the one being
// consumed (its own warp waits for every warp to release a stage before refilling it); each
// warp releases a stage after its MMAs on it.  A step is KB consecutive k-blocks of one tile.
// Counters run over the whole launch, so stage and phase follow from them:
// stage = count % STAGES, parity = (count / STAGES) & 1.
struct GpRing {
  uint64_t* full;
  uint64_t* empty;
  unsigned char* tiles;
  long long issued = 0, consumed = 0;
  int is = 0, cs = 0;            // stage of the next issue / consumption
  uint32_t iph = 0, cph = 0;     // their phase parities
};

// Stage layout: KB boxes of the A panel (rows I), then KB boxes of the B panel (rows J).
template <class C>
__device__ __forceinline__ bool gp_issue(GpRing& r, const CUtensorMap* map, int I, int J, int kb0,
                                         long long spins) {
  const int s = r.is;
  // refilling a stage: wait for every warp to have released its previous contents
  if (r.issued >= C::STAGES && !mbar_wait(r.empty + s, r.iph ^ 1u, spins)) return false;
  unsigned char* st = r.tiles + s * C::STAGE_BYTES;
  mbar_arrive_expect_tx(r.full + s, C::STAGE_BYTES);
#pragma unroll
  for (int b = 0; b < C::KB; ++b) {
    tma_load_2d(st + b * C::BOX_BYTES, map, (kb0 + b) * kGpK, I * C::BM, r.full + s);
    tma_load_2d(st + (C::KB + b) * C::BOX_BYTES, map, (kb0 + b) * kGpK, J * C::BM, r.full + s);
  }
  ++r.issued;
  if (++r.is == C::STAGES) { r.is = 0; r.iph ^= 1u; }
  return true;
}

// Position of a CTA in its sequence of ring steps: tile m (the CTA's m-th tile, (I, J)) and
// k-step kb; advanced one step at a time (one tri_inverse per tile).
struct GpCursor {
  int m = 0, kb = 0, I = 0, J = 0;
  __device__ __forceinline__ void start(int G) {
    m = kb = 0;
    tri_inverse(blockIdx.x, I, J);
    (void)G;
  }
  __device__ __forceinline__ void next(int kblocks, int G) {
    if (++kb == kblocks) {
      kb = 0;
      ++m;
      tri_inverse(blockIdx.x + (int64_t)m * G, I, J);
    }
  }
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
  const int nsteps = my_tiles * kblocks;  // ring steps of this CTA per product
  double* const buf0 = a.buf[0];
  double* const buf1 = a.buf[1];
  double t1 = a.t0[0], t2 = a.t0[1];
  int tail = -1, result = -1, cur = 0;
  const int g = lane >> 2, q = lane & 3;
  const int wm = warp / C::WGN, wn = warp % C::WGN;
  for (int it = a.it0;; ++it) {
    // ---- the decision of purify_fp64_loop, identical in every thread of every CTA ----
    if (!(fabs(t1) < INFINITY) || !(fabs(t2) < INFINITY)) { result = -1; break; }
    if (tail < 0 && fabs(t1 - t2) < kPurifyIdem) tail = kPurifyTail;
    if (fabs(t1 - t2) < kPurifyIdemFinal) tail = 0;
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
    GpCursor ic;  // thread 0: the next step to load
    if (threadIdx.x == 0 && nsteps > 0) {  // fill the ring with this product's first steps
      ic.start(G);
      for (int j = 0; j < C::STAGES && j < nsteps; ++j) {
        if (!gp_issue<C>(ring, map, ic.I, ic.J, ic.kb * C::KB, a.spins)) {
          s_abort = 1;
          atomicExch(a.bar.err, 1);
          break;
        }
        ic.next(kblocks, G);
      }
    }
    double acc[C::FM][C::FN][2];
    GpCursor cc;  // the step being consumed
    if (nsteps > 0) cc.start(G);
    for (int j = 0; j < nsteps && !s_abort; ++j) {
      const int I = cc.I, J = cc.J, kb = cc.kb;
      if (kb == 0) {
#pragma unroll
        for (int fm = 0; fm < C::FM; ++fm)
#pragma unroll
          for (int fn = 0; fn < C::FN; ++fn) acc[fm][fn][0] = acc[fm][fn][1] = 0.0;
      }
      const int s = ring.cs;
      if (!mbar_wait(ring.full + s, ring.cph, a.spins)) {
        s_abort = 1;
        atomicExch(a.bar.err, 1);
        break;
      }
#pragma unroll 1
      for (int kx = 0; kx < 2 * C::KB; ++kx) {
        const int box = kx >> 1, kk = kx & 1;
        const unsigned char* As = ring.tiles + s * C::STAGE_BYTES + box * C::BOX_BYTES;
        const unsigned char* Bs = As + C::KB * C::BOX_BYTES;
        // lane (g, q) reads the 16-byte chunk 2q + kk of its fragment row (doubles 4q + 2kk and
        // 4q + 2kk + 1), stored at chunk ^ (row % 8) = chunk ^ g.  Even chunks for kk = 0, odd
        // for kk = 1: the two rows g = 2i, 2i + 1 of a quarter-warp then hit 8 distinct 16-byte
        // bank groups (no conflict).  A and B use the same k order, so the sum is unchanged.
        const int chunk = ((2 * q + kk) ^ g) * 16;
        double2 b[C::FN];
#pragma unroll
        for (int fn = 0; fn < C::FN; ++fn)
          b[fn] = *reinterpret_cast<const double2*>(Bs + (wn * C::WN + fn * 8 + g) * 128 + chunk);
#pragma unroll
        for (int fm = 0; fm < C::FM; ++fm) {
          const double2 av =
              *reinterpret_cast<const double2*>(As + (wm * C::WM + fm * 8 + g) * 128 + chunk);
#pragma unroll
          for (int fn = 0; fn < C::FN; ++fn)
            dmma884(acc[fm][fn][0], acc[fm][fn][1], av.x, b[fn].x);
#pragma unroll
          for (int fn = 0; fn < C::FN; ++fn)
            dmma884(acc[fm][fn][0], acc[fm][fn][1], av.y, b[fn].y);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(ring.empty + s);
      ++ring.consumed;
      if (++ring.cs == C::STAGES) { ring.cs = 0; ring.cph ^= 1u; }
      cc.next(kblocks, G);
      if (threadIdx.x == 0 && j + C::STAGES < nsteps) {
        if (!gp_issue<C>(ring, map, ic.I, ic.J, ic.kb * C::KB, a.spins)) {
          s_abort = 1;
          atomicExch(a.bar.err, 1);
        }
        ic.next(kblocks, G);
      }
      if (kb != kblocks - 1) continue;
      // ---- epilogue of the tile: branch, lower-triangle elements and their mirrors ----
#pragma unroll
      for (int fm = 0; fm < C::FM; ++fm) {
        const int r = I * C::BM + wm * C::WM + fm * 8 + g;
#pragma unroll
        for (int fn = 0; fn < C::FN; ++fn) {
          const int c = J * C::BM + wn * C::WN + fn * 8 + 2 * q;
          if (r < c) continue;  // only on diagonal tiles: both elements above the diagonal
          double2 v;
          if (sq) {
            v = make_double2(acc[fm][fn][0], acc[fm][fn][1]);
          } else {
            const double2 x = __ldcg(reinterpret_cast<const double2*>(X + (int64_t)r * np + c));
            v = make_double2(fma(2.0, x.x, -acc[fm][fn][0]), fma(2.0, x.y, -acc[fm][fn][1]));
          }
          if (r > c) {  // (r, c) below the diagonal; (r, c + 1) below it or on it
            __stcg(reinterpret_cast<double2*>(Y + (int64_t)r * np + c), v);
            __stcg(Y + (int64_t)c * np + r, v.x);
            s2 = fma(2.0 * v.x, v.x, s2);
            if (r > c + 1) {
              __stcg(Y + (int64_t)(c + 1) * np + r, v.y);
              s2 = fma(2.0 * v.y, v.y, s2);
            } else {
              s1 += v.y;
              s2 = fma(v.y, v.y, s2);
            }
          } else {  // r == c: the diagonal element only (c + 1 is above it)
            __stcg(Y + (int64_t)r * np + c, v.x);
            s1 += v.x;
            s2 = fma(v.x, v.x, s2);
          }
        }
      }
    }
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
