// TF32 tensor-core products (tcgen05.mma kind::tf32, accumulators in tensor memory) for the
// FP32 phase of the mixed-precision purification: X kept split in two TF32 parts, hi = X with
// the low 13 mantissa bits cleared and lo = X - hi, and X^2 ~ hi hi^T + hi lo^T + lo hi^T (about
// 21 mantissa bits per product, the accuracy of an FP32 product).  Operands are 128-row panels
// of hi and lo, K-major, staged by TMA in the 128-byte swizzle.  Used by the whole-GPU loop
// (grid_purify32.cuh) and by one CTA per molecule (block_purify_tiles32 below, molecules above
// the shared-memory limit in a batch).
#pragma once
#include "dmma_tiles.cuh"

namespace sgb {

constexpr int kTfBM = 128;                  // tile rows = MMA M = MMA N
constexpr int kTfK = 32;                    // floats per k-block (one 128-byte swizzle row)
constexpr int kTfBox = kTfBM * 128;         // one panel part (hi or lo) of one k-block: 16 KB
constexpr int kTfStageBytes = 4 * kTfBox;   // A hi, A lo, B hi, B lo
constexpr int kTfTmemCols = 256;            // two 128-column FP32 accumulators

// Shared-memory matrix descriptor of a K-major operand in the 128-byte swizzle layout TMA
// writes: 8-row groups 1024 bytes apart (stride byte offset), descriptor version 1, swizzle
// mode 2 (128 B).  The k-slices of a 128-byte row are addressed by advancing the start address
// (the swizzle is applied to the absolute shared-memory address, as TMA applied it).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

// Splits v into its TF32 head and the FP32 remainder.
__device__ __forceinline__ void tf32_split(float v, float& h, float& l) {
  h = __uint_as_float(__float_as_uint(v) & 0xFFFFE000u);
  l = v - h;
}


// ---- one CTA, one molecule ---------------------------------------------------------------

constexpr int kBpTfStages = 2;  // 2 x 64 KB
constexpr size_t kBpRingBytes =
    1024 + (kBpRingFp64 > (size_t)kBpTfStages * kTfStageBytes ? kBpRingFp64
                                                               : (size_t)kBpTfStages * kTfStageBytes) +
    256;  // alignment, the stages, the barriers
// For these orders the FP32 phase's idempotency floor is near 1e-4 (n eigenvalues with FP32-level
// errors), so it hands over to FP64 at 1e-3, as the whole-GPU form does.
constexpr double kBpTf32Switch = 1e-3;

// The mixed form of block_purify_tiles for one CTA of 512 threads: X_0 from F in FP64 (slot X),
// rounded to FP32 into slot Y (set 1: one FP32 matrix, row stride n16 + 8 floats), then products
// on the tensor cores while tr(X - X^2) >= kBpTf32Switch -- warp 0 loads each k-block's two
// panels (one on a diagonal tile) by TMA into the hi parts of a ring stage, warps 2-3 split them
// in place into hi and lo (same swizzled offsets in the two parts), warp 1 issues the three MMAs
// per k-slice into one of two 128-column accumulators, warps 4-15 (one thread per tile row,
// three warps per row) read the accumulator and write the new X into the other set -- then X is
// widened to FP64 into the slot the last set does not hold and bp_fp64_loop finishes.  Keeping
// X in FP32 and splitting on chip halves the panel bytes each tile reads from memory (hi and lo
// both held in memory before): with every SM streaming its own molecule's panels this phase is
// bound by DRAM.  maps: [0] X slot FP64, [1] Y slot FP64, [2] set 0 FP32 (slot X), [4] set 1
// FP32 (slot Y), 128-row boxes of 32 floats; [3] and [5] are not used here.
template <int NT>
__device__ __noinline__ int block_purify_tiles32(const double* F, int n, int nocc, double* X,
                                                 double* Y, const CUtensorMap* maps,
                                                 unsigned char* ring_raw, double* lz, double* red,
                                                 double** Xout, long long spins) {
  static_assert(NT == 512, "warps 4-15 read the four tensor-memory lane quarters, three each");
  constexpr int NW = NT / 32;
  const int ld = purify_ld(n), n16 = purify_n16(n);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ volatile int s_abort;
  __shared__ uint32_t s_tmem;
  double t1, t2;
  purify_init<NT>(F, n, X, ld, lz, red, t1, t2);
  float* hs[2] = {reinterpret_cast<float*>(X), reinterpret_cast<float*>(Y)};
  {  // X_0 (FP64) -> set 1 (FP32) with its sums
    double s1 = 0.0, s2 = 0.0;
    float* H = hs[1];
    for (int64_t t = threadIdx.x; t < (int64_t)n16 * n16; t += NT) {
      const int r = (int)(t / n16), c = (int)(t - (int64_t)r * n16);
      const float v = (float)X[(int64_t)r * ld + c];
      H[(int64_t)r * ld + c] = v;
      const double x = (double)v;
      if (r == c) s1 += x;
      s2 = fma(x, x, s2);
    }
    block_sum2<NT>(s1, s2, red);
    t1 = s1;
    t2 = s2;
  }
  unsigned char* tiles = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(ring_raw) + 1023) & ~uintptr_t(1023));
  // the barriers sit past the stages of both this ring and the FP64 ring that follows
  // (bp_fp64_loop puts its own right after its stages), so the two never share an address
  static_assert(kBpTfStages * kTfStageBytes >= kBpRingFp64, "the FP64 ring is not larger");
  uint64_t* full = reinterpret_cast<uint64_t*>(tiles + kBpTfStages * kTfStageBytes + 128);
  uint64_t* empty = full + kBpTfStages;
  uint64_t* ready = empty + kBpTfStages;
  uint64_t* accf = ready + kBpTfStages;
  uint64_t* acce = accf + 2;
  uint64_t* drain = acce + 2;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kBpTfStages; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
      mbar_init(ready + s, 2);  // the two splitting warps
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf + b, 1);
      mbar_init(acce + b, 12);
    }
    mbar_init(drain, 1);
    mbar_fence_init();
    s_abort = 0;
  }
  if (warp == 1)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&s_tmem)),
                 "r"(kTfTmemCols));
  fence_proxy_async_global();  // set 1 is read by TMA
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = s_tmem;
  const int nt = (n16 + kTfBM - 1) / kTfBM, T = nt * (nt + 1) / 2;
  const int kblocks = (n16 + kTfK - 1) / kTfK;
  const uint32_t idesc = umma_idesc_tf32(kTfBM, kTfBM);
  long long issued = 0, split = 0, consumed = 0, mma_tiles = 0, epi_tiles = 0;
  int cur = 1, it = 0;
  bool ok = true;
  for (;; ++it) {
    if (!(fabs(t1) < INFINITY) || !(fabs(t2) < INFINITY) || it == kPurifyMaxIter) {
      ok = false;
      break;
    }
    if (t1 - t2 < kBpTf32Switch) break;
    const double n_o = (double)nocc;
    const bool sq = fabs(t2 - n_o) < fabs(2.0 * t1 - t2 - n_o);
    const CUtensorMap* mx = maps + 2 + 2 * cur;
    const float* Xs = hs[cur];
    float* Ys = hs[cur ^ 1];
    double s1 = 0.0, s2 = 0.0;
    if (warp == 0) {
      if (lane == 0) {  // ---- loader ----
        for (int t = 0; t < T && !s_abort; ++t) {
          int I, J;
          tri_inverse(t, I, J);
          for (int kb = 0; kb < kblocks; ++kb) {
            const int s = (int)(issued % kBpTfStages);
            if (issued >= kBpTfStages &&
                !mbar_wait(empty + s, (uint32_t)((issued / kBpTfStages - 1) & 1), spins)) {
              s_abort = 1;
              break;
            }
            unsigned char* st = tiles + s * kTfStageBytes;
            mbar_arrive_expect_tx(full + s, I == J ? kTfBox : 2 * kTfBox);
            tma_load_2d(st, mx, kb * kTfK, I * kTfBM, full + s);
            if (I != J) tma_load_2d(st + 2 * kTfBox, mx, kb * kTfK, J * kTfBM, full + s);
            ++issued;
          }
        }
      }
    } else if (warp == 2 || warp == 3) {
      // ---- split: each loaded FP32 part -> hi (in place) and lo (the next 16 KB) ----
      const int tid = threadIdx.x - 64;
      for (int t = 0; t < T && !s_abort; ++t) {
        int I, J;
        tri_inverse(t, I, J);
        const int parts = I == J ? 1 : 2;
        for (int kb = 0; kb < kblocks; ++kb) {
          const int s = (int)(split % kBpTfStages);
          if (!mbar_wait(full + s, (uint32_t)((split / kBpTfStages) & 1), spins)) {
            s_abort = 1;
            break;
          }
          unsigned char* st = tiles + s * kTfStageBytes;
          for (int p = 0; p < parts; ++p) {
            float4* hb = reinterpret_cast<float4*>(st + 2 * p * kTfBox);
            float4* lb = reinterpret_cast<float4*>(st + (2 * p + 1) * kTfBox);
#pragma unroll 4
            for (int q = tid; q < kTfBox / 16; q += 64) {
              const float4 v = hb[q];
              float4 h, l;
              tf32_split(v.x, h.x, l.x);
              tf32_split(v.y, h.y, l.y);
              tf32_split(v.z, h.z, l.z);
              tf32_split(v.w, h.w, l.w);
              hb[q] = h;
              lb[q] = l;
            }
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // read by the MMAs
          __syncwarp();
          if (lane == 0) mbar_arrive(ready + s);
          ++split;
        }
      }
    } else if (warp == 1) {
      if (lane == 0) {  // ---- MMA issue ----
        for (int t = 0; t < T && !s_abort; ++t) {
          int I, J;
          tri_inverse(t, I, J);
          const uint32_t boff = I == J ? 0u : 2u * kTfBox;  // a diagonal tile squares its panel
          const int b = (int)(mma_tiles & 1);
          const long long use = mma_tiles >> 1;
          if (use >= 1 && !mbar_wait(acce + b, (uint32_t)((use - 1) & 1), spins)) {
            s_abort = 1;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;");
          const uint32_t d = tmem + (uint32_t)(b * kTfBM);
          for (int kb = 0; kb < kblocks; ++kb) {
            const int s = (int)(consumed % kBpTfStages);
            if (!mbar_wait(ready + s, (uint32_t)((consumed / kBpTfStages) & 1), spins)) {
              s_abort = 1;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t base = smem_addr(tiles + s * kTfStageBytes);
#pragma unroll
            for (int ks = 0; ks < kTfK / 8; ++ks) {
              const uint32_t off = (uint32_t)ks * 32;
              const uint64_t ah = umma_desc_sw128(base + off);
              const uint64_t al = umma_desc_sw128(base + kTfBox + off);
              const uint64_t bh = umma_desc_sw128(base + boff + off);
              const uint64_t bl = umma_desc_sw128(base + boff + kTfBox + off);
              umma_tf32(d, ah, bh, idesc, (kb | ks) ? 1u : 0u);
              umma_tf32(d, ah, bl, idesc, 1u);
              umma_tf32(d, al, bh, idesc, 1u);
            }
            umma_commit(empty + s);
            ++consumed;
          }
          if (s_abort) break;
          umma_commit(accf + b);
          ++mma_tiles;
        }
      }
    } else if (warp >= 4) {
      // ---- epilogue: warps 4-15, one thread per tile row (tensor-memory lane 32 (warp & 3) +
      // lane), three warps per lane quarter, each taking a third of the 16-column chunks ----
      const int quad = warp & 3;
      const int part = (warp - 4) >> 2;  // 0, 1, 2
      const int lr = 32 * quad + lane;
      for (int t = 0; t < T && !s_abort; ++t) {
        int I, J;
        tri_inverse(t, I, J);
        const int b = (int)(epi_tiles & 1);
        if (!mbar_wait(accf + b, (uint32_t)((epi_tiles >> 1) & 1), spins)) {
          s_abort = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        const int r = I * kTfBM + lr;
        const int64_t row = (int64_t)r * ld;
        const uint32_t taddr = tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)(b * kTfBM);
#pragma unroll 1
        for (int c0 = 16 * part; c0 < kTfBM; c0 += 48) {
          uint32_t v[16];
          tmem_ld16(taddr + (uint32_t)c0, v);  // every lane: the load is warp-collective
          const int cb = J * kTfBM + c0;
          if (r >= n16 || cb >= n16 || r < cb) continue;  // past the matrix / above the diagonal
#pragma unroll
          for (int g4 = 0; g4 < 4; ++g4) {
            const int c = cb + 4 * g4;  // n16 is a multiple of 16: c .. c + 3 all inside
            // the old X only enters the 2X - X^2 branch
            float old[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            if (!sq) {
              const float4 o = __ldcg(reinterpret_cast<const float4*>(Xs + row + c));
              old[0] = o.x; old[1] = o.y; old[2] = o.z; old[3] = o.w;
            }
            float xn[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const float d2 = __uint_as_float(v[4 * g4 + e]);
              xn[e] = sq ? d2 : fmaf(2.0f, old[e], -d2);
            }
            // the thread's own row: one 16-byte store when the four columns are all at or below
            // the diagonal (a lane per row, so 4-byte stores would each take a sector); the
            // mirror column: lanes hold consecutive rows, so those stores coalesce
            if (r >= c + 3)
              __stcg(reinterpret_cast<float4*>(Ys + row + c), make_float4(xn[0], xn[1], xn[2], xn[3]));
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const int ce = c + e;
              if (r < ce) continue;
              if (r < c + 3) __stcg(Ys + row + ce, xn[e]);
              const double x = (double)xn[e];
              if (r == ce) {
                s1 += x;
                s2 = fma(x, x, s2);
              } else {
                __stcg(Ys + (int64_t)ce * ld + r, xn[e]);
                s2 = fma(2.0 * x, x, s2);
              }
            }
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncwarp();
        if (lane == 0) mbar_arrive(acce + b);
        ++epi_tiles;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    double* pr = red + 32 * (it & 1);
    if (lane == 0) { pr[warp] = s1; pr[16 + warp] = s2; }
    fence_proxy_async_global();  // the new set is read by TMA in the next product
    __syncthreads();
    if (s_abort) {
      ok = false;
      break;
    }
    s1 = 0.0;
    s2 = 0.0;
#pragma unroll
    for (int k = 0; k < NW; ++k) { s1 += pr[k]; s2 += pr[16 + k]; }
    t1 = s1;
    t2 = s2;
    cur ^= 1;
  }
  if (s_abort) {
    // loads and MMAs still in flight write this CTA's shared and tensor memory: wait for them
    // (bounded) before the memory is given back
    if (warp == 0 && lane == 0)
      for (long long c = issued - kBpTfStages; c < issued; ++c)
        if (c >= 0)
          mbar_wait(full + (int)(c % kBpTfStages), (uint32_t)((c / kBpTfStages) & 1), kMbarSpins);
    if (warp == 1 && lane == 0) {
      umma_commit(drain);
      mbar_wait(drain, 0, kMbarSpins);
    }
  } else if (warp == 0 && lane == 0) {
    // the MMAs' last releases of the stages (tcgen05.commit arrivals nobody waited for): let
    // them land before the barriers are invalidated
    for (long long c = issued - kBpTfStages; c < issued; ++c)
      if (c >= 0)
        mbar_wait(empty + (int)(c % kBpTfStages), (uint32_t)((c / kBpTfStages) & 1), kMbarSpins);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTfTmemCols));
  if (threadIdx.x == 0) {
    for (int s = 0; s < kBpTfStages; ++s) {
      asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(full + s)));
      asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(empty + s)));
      asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(ready + s)));
    }
    for (int b = 0; b < 2; ++b) {
      asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(accf + b)));
      asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(acce + b)));
    }
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(drain)));
  }
  __syncthreads();
  if (!ok) {
    *Xout = X;
    return -1;
  }
  // ---- widen the last set into the other slot (FP64) and finish in FP64 ----
  double* Xd = cur ? X : Y;  // the slot that does not hold set `cur`
  double* Yd = cur ? Y : X;
  const CUtensorMap* mXd = cur ? maps : maps + 1;
  const CUtensorMap* mYd = cur ? maps + 1 : maps;
  {
    const float* H = hs[cur];
    double s1 = 0.0, s2 = 0.0;
    for (int64_t t = threadIdx.x; t < (int64_t)n16 * n16; t += NT) {
      const int r = (int)(t / n16), c = (int)(t - (int64_t)r * n16);
      const int64_t a = (int64_t)r * ld + c, bb = (int64_t)c * ld + r;
      const double v = 0.5 * ((double)H[a] + (double)H[bb]);
      Xd[a] = v;
      if (r == c) s1 += v;
      s2 = fma(v, v, s2);
    }
    block_sum2<NT>(s1, s2, red);
    t1 = s1;
    t2 = s2;
  }
  return bp_fp64_loop<NT>(Xd, Yd, mXd, mYd, n, nocc, ring_raw, red, Xout, spins, it, t1, t2,
                          true);
}

}  // namespace sgb
