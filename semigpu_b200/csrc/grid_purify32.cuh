// Mixed precision on the whole GPU: the FP32 phase of the purification recursion (grid_purify.cuh)
// on the 5th-generation tensor cores, as one persistent cooperative launch.  X is kept split in
// two TF32 parts, hi = X with the low 13 mantissa bits cleared and lo = X - hi, so that
// X^2 ~ hi hi^T + hi lo^T + lo hi^T (three tcgen05.mma kind::tf32 per k-slice, FP32 accumulation
// in tensor memory): about 21 mantissa bits per product, the accuracy of an FP32 product.  The
// phase ends when tr(X - X^2) falls below the switch point; X is then widened to FP64 and the
// FP64 loop finishes the recursion, so the density keeps FP64 idempotency.
//
// Tiles are 128 x 128 (MMA M = N = 128) over the lower triangle, dealt round-robin to the CTAs.
// Per CTA: warp 0 loads (TMA, 128-byte swizzle, K-major: one k-block = 32 floats per row of
// the A-panel hi / lo and B-panel hi / lo boxes, 64 KB per ring stage); warp 1 issues the MMAs
// (one thread) into one of two 128-column accumulators and commits each stage back to the
// loader and each finished tile to the epilogue; warps 2-13 (one thread per tile row, the
// accumulator's tensor-memory lane, three warps per row splitting its columns) read the
// accumulator, apply X <- X^2 or 2X - X^2, write the new hi / lo (element and mirror) and add
// to the trace and squared-norm sums, while the MMAs of the next tile run into the other
// accumulator.  Products are separated by a grid barrier.
//
// Every wait is bounded (the context's wait limit); on a timeout the CTA waits (bounded) for
// its loads and MMAs in flight, gives its tensor memory back and the launch reports -2.
#pragma once
#include "grid_purify.cuh"
#include "tf32_tiles.cuh"

namespace sgb {

constexpr int kTfStages = 3;
// warp 0 loads, warp 1 issues the MMAs, warps 2-13 run the epilogue: three per quarter of the
// accumulator's tensor-memory lanes (a warp may read only the quarter warp % 4), each taking a
// third of the tile's 16-column chunks
constexpr int kTfThreads = 448;
constexpr int kTfEpiWarps = 12;
constexpr size_t kTfSmem = 1024 + (size_t)kTfStages * kTfStageBytes + 256;

struct GridPurify32Args {
  int np;              // padded order (multiple of 128), row stride of every part
  int nocc;
  float* hi[2];        // two sets of (hi, lo); X_0 in set 0
  float* lo[2];
  double* partial;     // 2 (product parity) x 2 (sums) x gridDim
  const double* t0;    // tr X_0, ||X_0||^2 (FP64)
  int* result;         // [0] products done when the phase ended (>= 0), -1 (non-finite, no
                       // convergence), -2 (a wait gave up); [1] the set holding X
  GridBarrier bar;
  long long spins;
  double switch_at;    // the phase ends when tr(X - X^2) < switch_at
};

__global__ void __launch_bounds__(kTfThreads, 1)
    k_grid_purify32(const __grid_constant__ CUtensorMap mh0, const __grid_constant__ CUtensorMap ml0,
                    const __grid_constant__ CUtensorMap mh1, const __grid_constant__ CUtensorMap ml1,
                    GridPurify32Args a) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* tiles = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(tiles + kTfStages * kTfStageBytes);
  uint64_t* empty = full + kTfStages;
  uint64_t* accf = empty + kTfStages;  // accumulator b complete (MMA -> epilogue)
  uint64_t* acce = accf + 2;           // accumulator b read (epilogue -> MMA)
  uint64_t* drain = acce + 2;          // the MMA thread's last commit (abort path)
  uint32_t* tslot = reinterpret_cast<uint32_t*>(drain + 1);
  __shared__ double red[2][kTfThreads / 32 + 1];
  __shared__ volatile int s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kTfStages; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf + b, 1);
      mbar_init(acce + b, kTfEpiWarps);
    }
    mbar_init(drain, 1);
    mbar_fence_init();
    s_abort = 0;
    tma_prefetch_map(&mh0);
    tma_prefetch_map(&ml0);
    tma_prefetch_map(&mh1);
    tma_prefetch_map(&ml1);
  }
  if (warp == 1)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(tslot)),
                 "r"(kTfTmemCols));
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tslot;

  const int np = a.np, nt = np / kTfBM, T = nt * (nt + 1) / 2, kblocks = np / kTfK;
  const int G = gridDim.x;
  const int my_tiles = (int)blockIdx.x < T ? (T - 1 - (int)blockIdx.x) / G + 1 : 0;
  float* const hi0 = a.hi[0];
  float* const hi1 = a.hi[1];
  float* const lo0 = a.lo[0];
  float* const lo1 = a.lo[1];
  const uint32_t idesc = umma_idesc_tf32(kTfBM, kTfBM);
  double t1 = a.t0[0], t2 = a.t0[1];
  int result = -1, cur = 0;
  long long issued = 0, consumed = 0;  // loader: stages issued; MMA thread: stages consumed
  long long mma_tiles = 0, epi_tiles = 0;
  auto fail = [&]() {
    s_abort = 1;
    atomicExch(a.bar.err, 1);
  };
  for (int it = 0;; ++it) {
    if (!(fabs(t1) < INFINITY) || !(fabs(t2) < INFINITY)) { result = -1; break; }
    if (t1 - t2 < a.switch_at) { result = it; break; }
    if (it == kPurifyMaxIter) { result = -1; break; }
    const double n_o = (double)a.nocc;
    const bool sq = fabs(t2 - n_o) < fabs(2.0 * t1 - t2 - n_o);
    const CUtensorMap* mh = cur ? &mh1 : &mh0;
    const CUtensorMap* ml = cur ? &ml1 : &ml0;
    const float* Xh = cur ? hi1 : hi0;
    const float* Xl = cur ? lo1 : lo0;
    float* Yh = cur ? hi0 : hi1;
    float* Yl = cur ? lo0 : lo1;
    double s1 = 0.0, s2 = 0.0;
    if (warp == 0) {
      // ---- loader ----
      if (lane == 0) {
        for (int m = 0; m < my_tiles && !s_abort; ++m) {
          int I, J;
          tri_inverse(blockIdx.x + (int64_t)m * G, I, J);
          for (int kb = 0; kb < kblocks; ++kb) {
            const int s = (int)(issued % kTfStages);
            if (issued >= kTfStages &&
                !mbar_wait(empty + s, (uint32_t)((issued / kTfStages - 1) & 1), a.spins)) {
              fail();
              break;
            }
            unsigned char* st = tiles + s * kTfStageBytes;
            mbar_arrive_expect_tx(full + s, kTfStageBytes);
            tma_load_2d(st, mh, kb * kTfK, I * kTfBM, full + s);
            tma_load_2d(st + kTfBox, ml, kb * kTfK, I * kTfBM, full + s);
            tma_load_2d(st + 2 * kTfBox, mh, kb * kTfK, J * kTfBM, full + s);
            tma_load_2d(st + 3 * kTfBox, ml, kb * kTfK, J * kTfBM, full + s);
            ++issued;
          }
        }
      }
    } else if (warp == 1) {
      // ---- MMA issue ----
      if (lane == 0) {
        for (int m = 0; m < my_tiles && !s_abort; ++m) {
          const int b = (int)(mma_tiles & 1);
          const long long use = mma_tiles >> 1;
          if (use >= 1 && !mbar_wait(acce + b, (uint32_t)((use - 1) & 1), a.spins)) {
            fail();
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;");
          const uint32_t d = tmem + (uint32_t)(b * kTfBM);
          bool ok = true;
          for (int kb = 0; kb < kblocks; ++kb) {
            const int s = (int)(consumed % kTfStages);
            if (!mbar_wait(full + s, (uint32_t)((consumed / kTfStages) & 1), a.spins)) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t base = smem_addr(tiles + s * kTfStageBytes);
#pragma unroll
            for (int ks = 0; ks < kTfK / 8; ++ks) {  // k-slices of 8 TF32 = 32 bytes
              const uint32_t off = (uint32_t)ks * 32;
              const uint64_t ah = umma_desc_sw128(base + off);
              const uint64_t al = umma_desc_sw128(base + kTfBox + off);
              const uint64_t bh = umma_desc_sw128(base + 2 * kTfBox + off);
              const uint64_t bl = umma_desc_sw128(base + 3 * kTfBox + off);
              const uint32_t acc = (kb | ks) ? 1u : 0u;
              umma_tf32(d, ah, bh, idesc, acc);
              umma_tf32(d, ah, bl, idesc, 1u);
              umma_tf32(d, al, bh, idesc, 1u);
            }
            umma_commit(empty + s);  // the stage is free once these MMAs have read it
            ++consumed;
          }
          if (!ok) {
            fail();
            break;
          }
          umma_commit(accf + b);
          ++mma_tiles;
        }
      }
    } else {
      // ---- epilogue: warps 2-13, one thread per tile row (tensor-memory lane), a third of the
      // column chunks per warp ----
      const int quad = warp & 3;  // the tensor-memory lanes this warp may read: 32 quad ..
      const int part = (warp - 2) >> 2;  // 0, 1, 2
      const int lr = 32 * quad + lane;
      for (int m = 0; m < my_tiles && !s_abort; ++m) {
        int I, J;
        tri_inverse(blockIdx.x + (int64_t)m * G, I, J);
        const int b = (int)(epi_tiles & 1);
        if (!mbar_wait(accf + b, (uint32_t)((epi_tiles >> 1) & 1), a.spins)) {
          fail();
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        const int r = I * kTfBM + lr;
        const int64_t row = (int64_t)r * np;
        const uint32_t taddr = tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)(b * kTfBM);
        const bool diag = I == J;
#pragma unroll 1
        for (int c0 = 16 * part; c0 < kTfBM; c0 += 48) {
          uint32_t v[16];
          tmem_ld16(taddr + (uint32_t)c0, v);
          const int cb = J * kTfBM + c0;
          if (diag && r < cb) continue;  // the whole chunk above the diagonal
#pragma unroll
          for (int g4 = 0; g4 < 4; ++g4) {
            const int c = cb + 4 * g4;
            // the old X only enters the 2X - X^2 branch
            float old[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            if (!sq) {
              const float4 oh = __ldcg(reinterpret_cast<const float4*>(Xh + row + c));
              const float4 ol = __ldcg(reinterpret_cast<const float4*>(Xl + row + c));
              old[0] = oh.x + ol.x; old[1] = oh.y + ol.y; old[2] = oh.z + ol.z; old[3] = oh.w + ol.w;
            }
            float nh[4], nl[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const float d2 = __uint_as_float(v[4 * g4 + e]);
              const float nv = sq ? d2 : fmaf(2.0f, old[e], -d2);
              tf32_split(nv, nh[e], nl[e]);
            }
            if (r > c + 3) {  // all four below the diagonal
              __stcg(reinterpret_cast<float4*>(Yh + row + c), make_float4(nh[0], nh[1], nh[2], nh[3]));
              __stcg(reinterpret_cast<float4*>(Yl + row + c), make_float4(nl[0], nl[1], nl[2], nl[3]));
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                __stcg(Yh + (int64_t)(c + e) * np + r, nh[e]);
                __stcg(Yl + (int64_t)(c + e) * np + r, nl[e]);
                const double x = (double)nh[e] + (double)nl[e];
                s2 = fma(2.0 * x, x, s2);
              }
            } else {
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                const int ce = c + e;
                if (r < ce) continue;
                __stcg(Yh + row + ce, nh[e]);
                __stcg(Yl + row + ce, nl[e]);
                const double x = (double)nh[e] + (double)nl[e];
                if (r == ce) {
                  s1 += x;
                  s2 = fma(x, x, s2);
                } else {
                  __stcg(Yh + (int64_t)ce * np + r, nh[e]);
                  __stcg(Yl + (int64_t)ce * np + r, nl[e]);
                  s2 = fma(2.0 * x, x, s2);
                }
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
      for (int w = 0; w < kTfThreads / 32; ++w) { b1 += red[0][w]; b2 += red[1][w]; }
      __stcg(part + blockIdx.x, b1);
      __stcg(part + G + blockIdx.x, b2);
    }
    fence_proxy_async_global();  // the new hi / lo are read by TMA in the next product
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
      if (lane == 0) { red[0][kTfThreads / 32] = u1; red[1][kTfThreads / 32] = u2; }
    }
    __syncthreads();
    t1 = red[0][kTfThreads / 32];
    t2 = red[1][kTfThreads / 32];
    cur ^= 1;
    __syncthreads();
  }
  if (result == -2) {
    // loads and MMAs still in flight write this CTA's shared and tensor memory: wait for them
    // (bounded) before the memory is given back
    if (threadIdx.x == 0)
      for (long long c = issued - kTfStages; c < issued; ++c)
        if (c >= 0) mbar_wait(full + (int)(c % kTfStages), (uint32_t)((c / kTfStages) & 1), kMbarSpins);
    if (warp == 1 && lane == 0) {
      umma_commit(drain);
      mbar_wait(drain, 0, kMbarSpins);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTfTmemCols));
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.result[0] = result;
    a.result[1] = cur;
  }
}

// X_0 = (hi I - F) / (hi - lo) split into TF32 hi / lo parts (padded np x np, zero padding);
// the sums of X_0 (as hi + lo) in FP64.
__global__ void k_gp_init32(int n, int np, const double* __restrict__ F, const double* lohi,
                            float* H, float* L, double* partial, unsigned* count, double* out) {
  const double lo = lohi[0], hi = lohi[1], inv = 1.0 / (hi - lo);
  const int64_t nn = (int64_t)np * np;
  double s1 = 0.0, s2 = 0.0;
  for (int64_t t = gtid(); t < nn; t += gstride()) {
    const int64_t i = t / np, j = t - i * np;
    float h = 0.0f, l = 0.0f;
    if (i < n && j < n) {
      tf32_split((float)(((i == j ? hi : 0.0) - F[i * n + j]) * inv), h, l);
      const double x = (double)h + (double)l;
      if (i == j) s1 += x;
      s2 = fma(x, x, s2);
    }
    H[t] = h;
    L[t] = l;
  }
  finalize_sums2(s1, s2, partial, count, out);
}

// X = hi + lo (FP32 parts, stride np32) widened into the padded FP64 buffer (stride np64),
// symmetrised; the sums of k_gp_init.
__global__ void k_gp_widen_split(int n, int np32, const float* __restrict__ H,
                                 const float* __restrict__ L, int np64, double* X,
                                 double* partial, unsigned* count, double* out) {
  const int64_t nn = (int64_t)np64 * np64;
  double s1 = 0.0, s2 = 0.0;
  for (int64_t t = gtid(); t < nn; t += gstride()) {
    const int64_t i = t / np64, j = t - i * np64;
    double v = 0.0;
    if (i < n && j < n) {
      const int64_t a = i * np32 + j, b = j * np32 + i;
      v = 0.5 * (((double)H[a] + (double)L[a]) + ((double)H[b] + (double)L[b]));
      if (i == j) s1 += v;
      s2 = fma(v, v, s2);
    }
    X[t] = v;
  }
  finalize_sums2(s1, s2, partial, count, out);
}

}  // namespace sgb
