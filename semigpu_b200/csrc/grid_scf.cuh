// Grid-wide kernels for one large molecule (nao above what one CTA's shared memory holds):
// the same per-task device code as the CTA path, spread over the whole GPU, with the SCF loop
// driven from the host.  The eigensolver is the same column-pair Jacobi on (V, G = F V), run as
// one cooperative launch per eigensolve: every warp of the grid takes column pairs of a round
// and the rounds are separated by a grid barrier.
#pragma once
#include "batch_scf.cuh"
#include "scf_block.cuh"

namespace sgb {

// ------------------------------------------------------------------------------------------
// Grid barrier for a cooperative launch (all blocks co-resident).  Sense by generation count;
// every wait is bounded: after `spins` polls the block records a timeout in *err and returns
// false, and every block leaves at its next barrier.  With co-residency guaranteed by the
// cooperative launch the bound is never reached in normal operation.  `expected` is the number
// of arrivals that completes a barrier (0: the grid's block count).
struct GridBarrier {
  unsigned* count;
  unsigned* gen;
  int* err;
  long long spins;
  unsigned expected;
};

constexpr long long kBarrierSpins = 1LL << 26;  // x >= 64 ns sleep: several seconds

__device__ bool grid_barrier(GridBarrier b) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = b.gen;
    const unsigned g = *vgen;
    __threadfence();
    const unsigned arrived = atomicAdd(b.count, 1u) + 1u;
    if (arrived == (b.expected ? b.expected : gridDim.x)) {
      *b.count = 0u;
      __threadfence();
      atomicAdd(b.gen, 1u);
    } else {
      long long spins = 0;
      while (*vgen == g) {
        if (++spins > b.spins || *(volatile int*)b.err) {
          atomicExch(b.err, 1);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile int*)b.err == 0;
}

// One barrier expecting `expected` arrivals, for the wait-limit test: with more arrivals
// expected than the grid has blocks, every block gives up after b.spins polls and *b.err is
// set (no block waits longer than that).
__global__ void k_barrier_probe(GridBarrier b) { grid_barrier(b); }

__device__ __forceinline__ int64_t gtid() { return blockIdx.x * (int64_t)blockDim.x + threadIdx.x; }
__device__ __forceinline__ int64_t gstride() { return (int64_t)gridDim.x * blockDim.x; }

// ------------------------------------------------------------------------------------------
// Setup stages and the Fock build, one task per thread.

__global__ void k_grid_integrals(MolView m) {
  const int64_t np = tri(m.natoms);
  for (int64_t p = gtid(); p < np; p += gstride()) {
    int A, B;
    tri_inverse(p, A, B);
    write_pair_block(m, A, B);
  }
}

__global__ void k_grid_hcore(MolView m) {
  const int64_t nd = (int64_t)m.natoms * 10, np = tri(m.natoms);
  for (int64_t t = gtid(); t < nd + np; t += gstride()) {
    if (t < nd) {
      const int A = (int)(t / 10), pq = (int)(t % 10);
      if (m.slot[A] == 0 && pq) continue;
      hcore_diag_atom(m, A, pq);
    } else {
      int A, B;
      tri_inverse(t - nd, A, B);
      if (A != B) hcore_offdiag_pair(m, A, B);
    }
  }
}

__global__ void k_grid_guess(MolView m) {
  const int64_t np = tri(m.nao);
  for (int64_t t = gtid(); t < np; t += gstride()) m.P[t] = 0.0;
}

__global__ void k_grid_guess_diag(MolView m) {
  for (int64_t A = gtid(); A < m.natoms; A += gstride()) {
    const int s = m.slot[A], n = nao_of_slot(s), f = m.first[A];
    for (int k = 0; k < n; ++k) m.P[tri(f + k) + f + k] = (double)c_elem[s].core / n;
  }
}

__global__ void k_grid_pair_density(MolView m, double* wq) {
  for (int64_t t = gtid(); t < (int64_t)m.natoms * 10; t += gstride()) pair_density_task(m, wq, (int)t);
}

// block partial sums of a per-thread value (deterministic second pass in k_reduce_sum)
__device__ void write_block_partial(double v, double* partial) {
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (l == 0) partial[blockIdx.x] = v;
  }
}

__global__ void k_grid_fock(MolView m, const double* wq, double* Ffull, double* partial) {
  const int64_t nd = (int64_t)m.natoms * 10, np = tri(m.natoms);
  double e = 0.0;
  for (int64_t t = gtid(); t < nd + np; t += gstride()) {
    if (t < nd) {
      e += fock_diag_task(m, wq, Ffull, m.nao, (int)t);
    } else {
      int A, B;
      tri_inverse(t - nd, A, B);
      if (A != B) e += fock_pair_task(m, Ffull, m.nao, A, B);
    }
  }
  write_block_partial(e, partial);
}

__global__ void k_grid_core_core(MolView m, double* partial) {
  double e = 0.0;
  for (int64_t p = gtid(); p < tri(m.natoms); p += gstride()) {
    int Bh, Al;
    tri_inverse(p, Bh, Al);
    if (Bh != Al) e += core_core_pair(m, Bh, Al);
  }
  write_block_partial(e, partial);
}

__global__ void k_reduce_sum(const double* partial, int n, double* out) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += partial[i];
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) *out = v;
  }
}

// E_el = 1/2 sum_ij P_ij (H_ij + F_ij) over the full symmetric matrices from their packed lower
// triangles (electronicenergy.cpp:12-36: the triangle twice, the diagonal once): block partials
// of (H + F) P weighted 1 off the diagonal and 1/2 on it; k_reduce_sum finishes the sum.
__global__ void k_energy_partials(int64_t np, const double* __restrict__ H,
                                  const double* __restrict__ F, const double* __restrict__ P,
                                  double* partial) {
  double e = 0.0;
  for (int64_t t = gtid(); t < np; t += gstride()) {
    int i, j;
    tri_inverse(t, i, j);
    const double v = (H[t] + F[t]) * P[t];
    e += i == j ? 0.5 * v : v;
  }
  write_block_partial(e, partial);
}

// ------------------------------------------------------------------------------------------
// Purification on the whole GPU: the recursion of purify.cuh for one large molecule runs in
// the device loops of grid_purify.cuh (FP64) and grid_purify32.cuh (the mixed form's FP32
// phase); the pieces here are the spectral bounds of F and the fixed-order finishing of block
// sums (deterministic).

// Block partials of (a, b); the last block to finish adds them up in a fixed order into
// out[0..1] (so the totals do not depend on which block is last) and resets *count, which must
// be 0 on entry.  Saves the second-pass launches between the products.
__device__ void finalize_sums2(double a, double b, double* partial, unsigned* count,
                               double* out) {
  write_block_partial(a, partial);
  __syncthreads();
  write_block_partial(b, partial + gridDim.x);
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(count, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double s1 = 0.0, s2 = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
    s1 += __ldcg(partial + i);
    s2 += __ldcg(partial + gridDim.x + i);
  }
  __shared__ double r1[32], r2[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) { r1[threadIdx.x >> 5] = s1; r2[threadIdx.x >> 5] = s2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t1 = 0.0, t2 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { t1 += r1[w]; t2 += r2[w]; }
    out[0] = t1;
    out[1] = t2;
    *count = 0;
  }
}

// Gershgorin bounds: per block, min over its rows of F_ii - r_i and max of F_ii + r_i
// (partial[2 blk], partial[2 blk + 1]); warp per row.
__global__ void k_pur_bounds(int n, const double* __restrict__ F, double* partial) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, nwb = blockDim.x >> 5;
  double lo = INFINITY, hi = -INFINITY;
  for (int64_t i = (int64_t)blockIdx.x * nwb + wib; i < n; i += (int64_t)gridDim.x * nwb) {
    const double* row = F + i * n;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += j == i ? 0.0 : fabs(row[j]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    lo = fmin(lo, row[i] - s);
    hi = fmax(hi, row[i] + s);
  }
  __shared__ double rlo[32], rhi[32];
  if (lane == 0) { rlo[wib] = lo; rhi[wib] = hi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < nwb; ++k) { lo = fmin(lo, rlo[k]); hi = fmax(hi, rhi[k]); }
    partial[2 * blockIdx.x] = lo;
    partial[2 * blockIdx.x + 1] = hi;
  }
}

__global__ void k_pur_bounds_reduce(const double* partial, int nb, double* lohi) {
  if (threadIdx.x == 0) {
    double lo = INFINITY, hi = -INFINITY;
    for (int b = 0; b < nb; ++b) { lo = fmin(lo, partial[2 * b]); hi = fmax(hi, partial[2 * b + 1]); }
    if (!(hi - lo > 1e-12)) hi = lo + 1.0;
    lohi[0] = lo;
    lohi[1] = hi;
  }
}






// Lanczos steps of the spectral bounds (purify.cuh), for one large molecule: the host keeps
// the coefficients and the loop; vectors q, q_prev, w of length n on the device.
__global__ void k_lz_start(int n, double* q, double* qp, double* partial) {
  double s = 0.0;
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const double v = lanczos_start((int)i);
    q[i] = v;
    qp[i] = 0.0;
    s = fma(v, v, s);
  }
  write_block_partial(s, partial);
}

__global__ void k_lz_scale(int n, double* q, const double* sumsq) {
  const double inv = 1.0 / sqrt(*sumsq);
  for (int64_t i = gtid(); i < n; i += gstride()) q[i] *= inv;
}

// w = F q - beta q_prev (warp per row); block partials of q.w and w.w
__global__ void k_lz_matvec(int n, const double* __restrict__ F, const double* q,
                            const double* qp, double beta, double* w, double* partial) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, nwb = blockDim.x >> 5;
  double qw = 0.0, ww = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * nwb + wib; i < n; i += (int64_t)gridDim.x * nwb) {
    const double* row = F + i * n;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s = fma(row[j], q[j], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const double wi = s - beta * qp[i];
    if (lane == 0) {
      w[i] = wi;
      qw = fma(q[i], wi, qw);
      ww = fma(wi, wi, ww);
    }
  }
  write_block_partial(qw, partial);
  __syncthreads();
  write_block_partial(ww, partial + gridDim.x);
}

__global__ void k_lz_update(int n, double* q, double* qp, const double* w, double alpha,
                            double rnb) {
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const double qi = q[i];
    qp[i] = qi;
    q[i] = (w[i] - alpha * qi) * rnb;
  }
}

// DIIS on the grid path (off by default): the error of step k is the commutator
// F_k P_k - P_k F_k (the basis is orthonormal in NDDO), formed from C = F P as C - C^T.
__global__ void k_commutator(int n, const double* __restrict__ C, double* E) {
  const int64_t nn = (int64_t)n * n;
  for (int64_t t = gtid(); t < nn; t += gstride()) {
    const int64_t j = t / n, i = t - j * n;
    E[t] = C[t] - C[j + i * n];
  }
}

__global__ void k_dot(int64_t nn, const double* __restrict__ a, const double* __restrict__ b,
                      double* partial) {
  double s = 0.0;
  for (int64_t t = gtid(); t < nn; t += gstride()) s = fma(a[t], b[t], s);
  write_block_partial(s, partial);
}

struct LinComb {
  const double* src[8];
  double c[8];
  int m;
};

__global__ void k_lincomb(int64_t nn, LinComb lc, double* out) {
  for (int64_t t = gtid(); t < nn; t += gstride()) {
    double v = 0.0;
    for (int k = 0; k < lc.m; ++k) v = fma(lc.c[k], lc.src[k][t], v);
    out[t] = v;
  }
}


// ------------------------------------------------------------------------------------------
// Dense pieces of the eigensolve (column-major n x n, ld n)

__global__ void k_grid_identity(int n, double* V, double* G, const double* F) {
  const int64_t nn = (int64_t)n * n;
  for (int64_t t = gtid(); t < nn; t += gstride()) {
    const int64_t j = t / n, i = t % n;
    V[t] = i == j ? 1.0 : 0.0;
    G[t] = F[t];
  }
}

// G = F V, 64x64 output tile per 256-thread CTA (4x4 per thread), K staged 16 at a time.
constexpr int kGemmTile = 64, kGemmK = 16;

__global__ void __launch_bounds__(256) k_grid_gemm(int n, const double* __restrict__ F,
                                                   const double* __restrict__ V,
                                                   double* __restrict__ G) {
  __shared__ double sF[kGemmK][kGemmTile + 1];  // F[i][k] for the tile's rows (F symmetric)
  __shared__ double sV[kGemmK][kGemmTile + 1];  // V[k][j] for the tile's columns
  const int i0 = blockIdx.x * kGemmTile, j0 = blockIdx.y * kGemmTile;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;  // 16 x 16 threads, 4 x 4 outputs
  double acc[4][4] = {};
  for (int k0 = 0; k0 < n; k0 += kGemmK) {
    for (int t = threadIdx.x; t < kGemmK * kGemmTile; t += blockDim.x) {
      const int kk = t / kGemmTile, r = t % kGemmTile;
      const int k = k0 + kk, i = i0 + r, j = j0 + r;
      // F is symmetric: F[i][k] = F[k][i] = F[k * n + i] (coalesced along i)
      sF[kk][r] = (k < n && i < n) ? F[(int64_t)k * n + i] : 0.0;
      sV[kk][r] = (k < n && j < n) ? V[(int64_t)j * n + k] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kGemmK; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = sF[kk][tx * 4 + r];
#pragma unroll
      for (int c = 0; c < 4; ++c) b[c] = sV[kk][ty * 4 + c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int c = 0; c < 4; ++c)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = i0 + tx * 4 + r, j = j0 + ty * 4 + c;
      if (i < n && j < n) G[(int64_t)j * n + i] = acc[r][c];
    }
}

// dval[i] = v_i . g_i, one warp per column
__global__ void k_grid_rayleigh(int n, const double* G, const double* V, double* dval) {
  const int64_t w = gtid() >> 5, nw = gstride() >> 5;
  const int lane = threadIdx.x & 31;
  for (int64_t i = w; i < n; i += nw) {
    double s = 0.0;
    for (int k = lane; k < n; k += 32) s = fma(G[i * n + k], V[i * n + k], s);
    s = warp_sum(s);
    if (lane == 0) dval[i] = s;
  }
}

__global__ void k_grid_split(int n, int nocc, const double* dval, int* occ, int* vir) {
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const int rank = ascending_rank(dval, n, (int)i);
    if (rank < nocc) occ[rank] = (int)i;
    else vir[rank - nocc] = (int)i;
  }
}

// flag[0] = 1 when max dval over occ + margin >= min dval over vir (one block)
__global__ void k_grid_crossing(int nocc, int nvir, const double* dval, const int* occ,
                                const int* vir, double margin, int* flag) {
  double hi = -INFINITY, lo = INFINITY;
  for (int i = threadIdx.x; i < nocc; i += blockDim.x) hi = fmax(hi, dval[occ[i]]);
  for (int i = threadIdx.x; i < nvir; i += blockDim.x) lo = fmin(lo, dval[vir[i]]);
  __shared__ double sh[64];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
  }
  if ((threadIdx.x & 31) == 0) { sh[threadIdx.x >> 5] = hi; sh[32 + (threadIdx.x >> 5)] = lo; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { hi = fmax(hi, sh[w]); lo = fmin(lo, sh[32 + w]); }
    flag[0] = !(hi + margin < lo);
  }
}

// P (packed) = 2 sum_k V[:, occ[k]] V[:, occ[k]]^T, 4x4 register tiles on the lower triangle;
// mixed with the previous P by the damping factor d when d > 0
__global__ void k_grid_density(int n, int nocc, const double* V, const int* occ, double* P,
                               double d) {
  const int tiles = (n + 3) >> 2;
  const int64_t ntile = (int64_t)tiles * (tiles + 1) / 2;
  for (int64_t t = gtid(); t < ntile; t += gstride()) {
    int ti, tj;
    tri_inverse(t, ti, tj);
    const int i0 = ti * 4, j0 = tj * 4;
    double acc[4][4] = {};
    for (int k = 0; k < nocc; ++k) {
      const double* col = V + (int64_t)occ[k] * n;
      double a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = i0 + r < n ? col[i0 + r] : 0.0;
#pragma unroll
      for (int c = 0; c < 4; ++c) b[c] = j0 + c < n ? col[j0 + c] : 0.0;
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int i = i0 + r, j = j0 + c;
        if (i < n && j <= i) {
          const double p = 2.0 * acc[r][c];
          P[tri(i) + j] = d > 0.0 ? fma(d, P[tri(i) + j] - p, p) : p;
        }
      }
  }
}

// eig[rank(i)] = dval[i] and, when T != nullptr, T[:, rank(i)] = V[:, i]
__global__ void k_grid_sorted_output(int n, const double* dval, const double* V, double* eig,
                                     double* T) {
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const int rank = ascending_rank(dval, n, (int)i);
    eig[rank] = dval[i];
    if (T)
      for (int r = 0; r < n; ++r) T[(int64_t)rank * n + r] = V[i * n + r];
  }
}

// ------------------------------------------------------------------------------------------
// Cooperative Jacobi on (V, G = F V).  Same pair schedules as block_jacobi_fv (full
// round-robin or bipartite); columns stay in global memory and are read twice per pair (dot
// products, then the rotation).  worst[sweep] receives the largest |A_pq| seen (as the bit
// pattern of a non-negative double, so atomicMax orders it); result[0] gets the sweep count or
// -1 (no convergence / non-finite) or -2 (barrier timeout).
struct GridJacobiArgs {
  int n;
  double* G;
  double* V;
  const int* grp_a;
  int na;
  const int* grp_b;
  int nb;
  double rot_abs, done_abs;
  int max_sweeps;
  unsigned long long* worst;  // max_sweeps entries, zeroed before the launch
  int* result;
  GridBarrier bar;
};

__global__ void __launch_bounds__(256) k_grid_jacobi(GridJacobiArgs a) {
  const int n = a.n;
  const int ne = n + (n & 1), m = ne - 1, n2 = ne / 2;
  const bool bip = a.grp_a != nullptr;
  const int rounds = bip ? a.nb : m, per_round = bip ? a.na : n2;
  const int64_t gw = gtid() >> 5, nw = gstride() >> 5;
  const int lane = threadIdx.x & 31;
  __shared__ double sworst[8];
  for (int sweep = 0; sweep < a.max_sweeps; ++sweep) {
    double worst = 0.0;
    for (int r = 0; r < rounds; ++r) {
      for (int64_t k = gw; k < per_round; k += nw) {
        int p, q;
        if (bip) {
          p = a.grp_a[k];
          int j = (int)k + r;
          if (j >= a.nb) j -= a.nb;
          q = a.grp_b[j];
        } else {
          rr_pair(r, (int)k, m, p, q);
          if (p >= n || q >= n) continue;
        }
        double* gp = a.G + (int64_t)p * n;
        double* gq = a.G + (int64_t)q * n;
        double* vp = a.V + (int64_t)p * n;
        double* vq = a.V + (int64_t)q * n;
        double app = 0.0, aqq = 0.0, apq = 0.0, aqp = 0.0;
        for (int i = lane; i < n; i += 32) {
          const double xg = gp[i], yg = gq[i], xv = vp[i], yv = vq[i];
          app = fma(xv, xg, app);
          aqq = fma(yv, yg, aqq);
          apq = fma(xv, yg, apq);
          aqp = fma(xg, yv, aqp);
        }
        warp_sum4(lane, app, aqq, apq, aqp);
        const double a_pq = 0.5 * (apq + aqp);
        if (!(fabs(a_pq) > a.rot_abs)) {
          if (a_pq != a_pq) worst = INFINITY;
          continue;
        }
        worst = fmax(worst, fabs(a_pq));
        const float num = (float)(2.0 * a_pq), den = (float)(aqq - app);
        float tf = num / (fabsf(den) + hypotf(den, num));
        if (den < 0.0f) tf = -tf;
        const double t = (double)tf;
        const double c = rsqrt(fma(t, t, 1.0)), s = c * t;
        for (int i = lane; i < n; i += 32) {
          const double xg = gp[i], yg = gq[i], xv = vp[i], yv = vq[i];
          gp[i] = c * xg - s * yg;
          gq[i] = s * xg + c * yg;
          vp[i] = c * xv - s * yv;
          vq[i] = s * xv + c * yv;
        }
      }
      if (!grid_barrier(a.bar)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) a.result[0] = -2;
        return;
      }
    }
    // sweep maximum over the grid
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) worst = fmax(worst, __shfl_xor_sync(0xffffffffu, worst, o));
    if (lane == 0) sworst[threadIdx.x >> 5] = worst;
    __syncthreads();
    if (threadIdx.x == 0) {
      double w = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) w = fmax(w, sworst[i]);
      atomicMax(a.worst + sweep, (unsigned long long)__double_as_longlong(w));
    }
    if (!grid_barrier(a.bar)) {
      if (blockIdx.x == 0 && threadIdx.x == 0) a.result[0] = -2;
      return;
    }
    const double w = __longlong_as_double((long long)*(volatile unsigned long long*)(a.worst + sweep));
    if (!(w < INFINITY)) {
      if (blockIdx.x == 0 && threadIdx.x == 0) a.result[0] = -1;
      return;
    }
    if (w < a.done_abs) {
      if (blockIdx.x == 0 && threadIdx.x == 0) a.result[0] = sweep + 1;
      return;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) a.result[0] = -1;
}

}  // namespace sgb
