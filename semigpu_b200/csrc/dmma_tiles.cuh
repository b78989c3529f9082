// FP64 tile products on the tensor cores for the purification recursion: X^2 of a symmetric X
// over the lower triangle of BM x BM tiles, the panels X[I-tile, :] and X[J-tile, :] (X^2 =
// X X^T) streamed through shared memory by TMA, the products as DMMA (mma.sync m8n8k4 f64)
// on register accumulators, and the update X <- X^2 or 2X - X^2 written to the partner buffer
// (element and mirror) with the trace and squared-norm sums.  Used by one CTA per molecule
// (batch_scf.cuh, molecules above the shared-memory limit) and by every CTA of the GPU for one
// molecule (grid_purify.cuh).
//
// The loads: k-blocks of 16 doubles (one 128-byte swizzled row per panel row; the swizzle spreads
// a warp's 16-byte fragment loads over all banks), KB of them per ring stage, in a ring of STAGES
// stages guarded by full / empty mbarriers.  Thread 0 issues the loads a ring ahead; every warp
// runs its MMAs on a stage and then releases it.
#pragma once
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
// Tile configurations of the whole-GPU loop (grid_purify.cuh).  Measured on C2000H2002 (10002 AOs, one FP64 SCF): the 128 x 128 tile with 8 warps of
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

// Position of a CTA in its sequence of ring steps: its m-th tile t0 + m * stride, (I, J), and
// k-step kb; advanced one step at a time (one tri_inverse per tile).
struct GpCursor {
  int m = 0, kb = 0, I = 0, J = 0, t0 = 0, stride = 1;
  __device__ __forceinline__ void start(int first, int step) {
    m = kb = 0;
    t0 = first;
    stride = step;
    tri_inverse(t0, I, J);
  }
  __device__ __forceinline__ void next(int kblocks) {
    if (++kb == kblocks) {
      kb = 0;
      ++m;
      tri_inverse(t0 + (int64_t)m * stride, I, J);
    }
  }
};


// One product over this CTA's tiles t_first, t_first + t_stride, ... (my_tiles of them, of the
// nt (nt + 1) / 2 lower-triangle tiles): X (row stride ld) -> Y for rows and columns below nw
// (the extent of the matrix; tiles past it read zeros and write nothing), branch sq (X^2) or
// 2X - X^2; s1 += trace, s2 += squared Frobenius norm of what this thread wrote.  The ring's
// barriers and counters carry over from call to call.  A wait that gives up sets *s_abort and
// *err and the product stops (the caller checks *s_abort).
template <class C>
__device__ __forceinline__ void gp_product(GpRing& ring, const CUtensorMap* map, const double* X,
                                           double* Y, int ld, int nw, int kblocks, int t_first,
                                           int t_stride, int my_tiles, bool sq, long long spins,
                                           volatile int* s_abort, int* err, double& s1,
                                           double& s2) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, q = lane & 3;
  const int wm = warp / C::WGN, wn = warp % C::WGN;
  const int nsteps = my_tiles * kblocks;
  GpCursor ic;  // thread 0: the next step to load
  if (threadIdx.x == 0 && nsteps > 0) {  // fill the ring with this product's first steps
    ic.start(t_first, t_stride);
    for (int j = 0; j < C::STAGES && j < nsteps; ++j) {
      if (!gp_issue<C>(ring, map, ic.I, ic.J, ic.kb * C::KB, spins)) {
        *s_abort = 1;
        atomicExch(err, 1);
        break;
      }
      ic.next(kblocks);
    }
  }
  double acc[C::FM][C::FN][2];
  GpCursor cc;  // the step being consumed
  if (nsteps > 0) cc.start(t_first, t_stride);
  for (int j = 0; j < nsteps && !*s_abort; ++j) {
    const int I = cc.I, J = cc.J, kb = cc.kb;
    if (kb == 0) {
#pragma unroll
      for (int fm = 0; fm < C::FM; ++fm)
#pragma unroll
        for (int fn = 0; fn < C::FN; ++fn) acc[fm][fn][0] = acc[fm][fn][1] = 0.0;
    }
    const int s = ring.cs;
    if (!mbar_wait(ring.full + s, ring.cph, spins)) {
      *s_abort = 1;
      atomicExch(err, 1);
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
    cc.next(kblocks);
    if (threadIdx.x == 0 && j + C::STAGES < nsteps) {
      if (!gp_issue<C>(ring, map, ic.I, ic.J, ic.kb * C::KB, spins)) {
        *s_abort = 1;
        atomicExch(err, 1);
      }
      ic.next(kblocks);
    }
    if (kb != kblocks - 1) continue;
    // ---- epilogue of the tile: branch, lower-triangle elements and their mirrors ----
#pragma unroll
    for (int fm = 0; fm < C::FM; ++fm) {
      const int r = I * C::BM + wm * C::WM + fm * 8 + g;
#pragma unroll
      for (int fn = 0; fn < C::FN; ++fn) {
        const int c = J * C::BM + wn * C::WN + fn * 8 + 2 * q;
        if (r < c || r >= nw) continue;  // above the diagonal (diagonal tiles) / past the matrix
        double2 v;
        if (sq) {
          v = make_double2(acc[fm][fn][0], acc[fm][fn][1]);
        } else {
          const double2 x = __ldcg(reinterpret_cast<const double2*>(X + (int64_t)r * ld + c));
          v = make_double2(fma(2.0, x.x, -acc[fm][fn][0]), fma(2.0, x.y, -acc[fm][fn][1]));
        }
        if (r > c) {  // (r, c) below the diagonal; (r, c + 1) below it or on it
          __stcg(reinterpret_cast<double2*>(Y + (int64_t)r * ld + c), v);
          __stcg(Y + (int64_t)c * ld + r, v.x);
          s2 = fma(2.0 * v.x, v.x, s2);
          if (r > c + 1) {
            __stcg(Y + (int64_t)(c + 1) * ld + r, v.y);
            s2 = fma(2.0 * v.y, v.y, s2);
          } else {
            s1 += v.y;
            s2 = fma(v.y, v.y, s2);
          }
        } else {  // r == c: the diagonal element only (c + 1 is above it)
          __stcg(Y + (int64_t)r * ld + c, v.x);
          s1 += v.x;
          s2 = fma(v.x, v.x, s2);
        }
      }
    }
  }
}

// ---- one CTA, one molecule: the recursion with X and its partner in global memory ----------

// 64 x 64 tiles, 16 warps of 16 x 16 (the batch kernel's 512 threads at its 128-register cap),
// 3 k-blocks per stage, 2 stages (96 KB).  148 alkanes of 164-902 AOs, one CTA each, FP64:
// 861 ms against 921 ms with 2 k-blocks x 3 stages and 897 ms with 4 x 2.
using BpCfg = GpCfg<64, 4, 4, 3, 2>;
constexpr size_t kBpRingFp64 = (size_t)BpCfg::STAGES * BpCfg::STAGE_BYTES;

// The FP64 recursion on X (n16 x n16, row stride n16 + 8, global memory) from product it0 with
// sums t1, t2, the products as TMA-staged DMMA tiles (gp_product) through the tensor maps mX /
// mY of X and its partner Y (64-row boxes of 16 doubles); ring_raw: kBpRingBytes of shared
// memory.  Returns the number of products and leaves the result in *Xout (X or Y), or -1 (no
// convergence, wrong trace, non-finite value, or a wait that gave up).
template <int NT>
__device__ __noinline__ int bp_fp64_loop(double* X, double* Y, const CUtensorMap* mX,
                                         const CUtensorMap* mY, int n, int nocc,
                                         unsigned char* ring_raw, double* red, double** Xout,
                                         long long spins, int it0, double t1, double t2,
                                         bool mixed_finish) {
  static_assert(NT == BpCfg::THREADS, "one warp per 16 x 16 warp tile of the 64 x 64 tile");
  constexpr int NW = NT / 32;
  const int ld = purify_ld(n), n16 = purify_n16(n);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ volatile int s_abort;
  __shared__ int s_err;
  GpRing ring;
  ring.tiles = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(ring_raw) + 1023) &
                                                ~uintptr_t(1023));
  ring.full = reinterpret_cast<uint64_t*>(ring.tiles + BpCfg::STAGES * BpCfg::STAGE_BYTES);
  ring.empty = ring.full + BpCfg::STAGES;
  if (threadIdx.x == 0) {
    for (int s = 0; s < BpCfg::STAGES; ++s) {
      mbar_init(ring.full + s, 1);
      mbar_init(ring.empty + s, BpCfg::WARPS);
    }
    mbar_fence_init();
    s_abort = 0;
    s_err = 0;
  }
  fence_proxy_async_global();  // X is read by TMA
  __syncthreads();
  const int nt = (n16 + BpCfg::BM - 1) / BpCfg::BM, T = nt * (nt + 1) / 2;
  const int kblocks = (n16 + kGpK * BpCfg::KB - 1) / (kGpK * BpCfg::KB);
  int tail = -1, result = -1;
  for (int it = it0;; ++it) {
    if (!(fabs(t1) < INFINITY) || !(fabs(t2) < INFINITY)) break;
    if (mixed_finish) {  // the mixed form: done at kMixedIdemFinal, no tail
      if (fabs(t1 - t2) < kMixedIdemFinal) tail = 0;
    } else {
      if (tail < 0 && fabs(t1 - t2) < kPurifyIdem) tail = kPurifyTail;
      if (fabs(t1 - t2) < kPurifyIdemFinal) tail = 0;
    }
    if (tail == 0) {
      if (fabs(t1 - (double)nocc) < kPurifyTraceTol) result = it;
      break;
    }
    if (tail > 0) --tail;
    if (it == kPurifyMaxIter) break;
    const double n_o = (double)nocc;
    const bool sq = fabs(t2 - n_o) < fabs(2.0 * t1 - t2 - n_o);
    double s1 = 0.0, s2 = 0.0;
    gp_product<BpCfg>(ring, mX, X, Y, ld, n16, kblocks, 0, 1, T, sq, spins, &s_abort, &s_err, s1,
                      s2);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    double* part = red + 32 * (it & 1);
    if (lane == 0) { part[warp] = s1; part[16 + warp] = s2; }
    fence_proxy_async_global();  // Y is read by TMA in the next product
    __syncthreads();             // Y and the partial sums complete
    if (s_abort) break;
    s1 = 0.0;
    s2 = 0.0;
#pragma unroll
    for (int k = 0; k < NW; ++k) { s1 += part[k]; s2 += part[16 + k]; }
    t1 = s1;
    t2 = s2;
    double* tx = X; X = Y; Y = tx;
    const CUtensorMap* tm = mX; mX = mY; mY = tm;
  }
  if (threadIdx.x == 0 && s_abort) {
    // loads still in flight land in this CTA's shared memory: wait for them (bounded)
    for (long long c = ring.consumed; c < ring.issued; ++c)
      mbar_wait(ring.full + (int)(c % BpCfg::STAGES), (uint32_t)((c / BpCfg::STAGES) & 1),
                kMbarSpins);
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int s = 0; s < BpCfg::STAGES; ++s) {
      asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(ring.full + s)));
      asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(ring.empty + s)));
    }
  __syncthreads();
  *Xout = X;
  return s_abort ? -1 : result;
}

// block_purify_global with the products as TMA-staged DMMA tiles (bp_fp64_loop): X_0 from F.
template <int NT>
__device__ __noinline__ int block_purify_tiles(const double* F, int n, int nocc, double* X,
                                               double* Y, const CUtensorMap* mapX,
                                               const CUtensorMap* mapY, unsigned char* ring_raw,
                                               double* lz, double* red, double** Xout,
                                               long long spins) {
  double t1, t2;
  purify_init<NT>(F, n, X, purify_ld(n), lz, red, t1, t2);
  return bp_fp64_loop<NT>(X, Y, mapX, mapY, n, nocc, ring_raw, red, Xout, spins, 0, t1, t2,
                          false);
}

}  // namespace sgb
