// Fock matrix and electronic energy of one molecule on one CTA, warp-cooperative.
//
// The reference builds F = Hcore + G(P) block by block (fockmatrix.cpp:32-53, the diagonal
// atom blocks with the Coulomb sum over every atom plus one-center exchange, the off-diagonal
// blocks with two-center exchange) and then E_el = 1/2 sum P (H + F)
// (electronicenergy.cpp:12-36).  Here the integral array is walked the way it is stored, so
// that every load is shared by a warp instead of one thread reading a 10 x 10 block alone
// (whose scattered loads made the L1 the bottleneck), and the work is cut into many similar
// pieces so that every warp has several independent loads in flight:
//   heavy-heavy blocks  dealt round-robin to the warps, one block at a time per warp with the
//                next block (integrals, and the P and H entries of its exchange block)
//                prefetched into registers.  The block is staged in shared memory; 16 lanes
//                form the 4 x 4 exchange block, 10 lanes the block's part of the Coulomb sum of
//                its row atom, J_A[pq] += sum_q (pq|q_B) w_B[q], and 10 lanes that of its column
//                atom, J_B[q] += sum_pq (pq|q_B) w_A[pq]; these 20 partial sums per block go to
//                scratch (xs) and are added in a fixed order afterwards;
//   blocks with a hydrogen  warp per atom: the hydrogen blocks of its row and of its column,
//                one block per lane;
//   diagonal     thread per (atom, pair): H + J - 1/2 one-center exchange.
// Every sum has a fixed order, so results do not depend on the schedule.
#pragma once
#include "scf_block.cuh"

namespace sgb {

constexpr int kFockStagePerWarp = 128;                 // one 10 x 10 block, padded
constexpr int kFockStage = 16 * kFockStagePerWarp;     // doubles, for up to 512 threads

// Scratch of the heavy-heavy partial Coulomb sums: 20 doubles per heavy atom pair, at most
// nao / 4 heavy atoms.
__host__ __device__ inline size_t fock_xx_doubles(int n) {
  const size_t q = (size_t)n / 4;
  return 20 * (q * (q + 1) / 2);
}

// Offset of block B within row A of the integral array.
__device__ __forceinline__ int64_t row_block(const MolView& m, bool hA, int B) {
  const int h = m.hb[B];
  return hA ? (int64_t)h * 100 + (int64_t)(B - h) * 10 : (int64_t)h * 10 + (B - h);
}

// Writes F(i, j), i > j, of an off-diagonal block; returns its energy term P (H + F).
__device__ __forceinline__ double put_offdiag(const MolView& m, double* Fs, int ld, int i, int j,
                                              double p, double g) {
  const int64_t ij = tri(i) + j;
  const double h = m.H[ij], fv = h - 0.5 * g;
  m.F[ij] = fv;
  if (Fs) {
    Fs[(int64_t)i * ld + j] = fv;
    Fs[(int64_t)j * ld + i] = fv;
  }
  return p * (h + fv);
}

// Heavy-heavy blocks k = warp, warp + nw, ... (k = a(a+1)/2 + b over heavy indices a >= b):
// exchange into F, partial Coulomb sums into xs[20 k ..].  Returns the energy share.
// The loop is issue-bound, so everything that does not change between blocks is hoisted: each
// lane's 8 exchange offsets into the staged block (the two half-warps split the 16 (lam, sig)
// terms of the same 4 x 4 output), its Coulomb row or column, and the pair indices (a, b),
// which advance by nw without a square root.
__device__ __noinline__ double fock_xx_blocks(const MolView& m, const int* hv, int nh,
                                              const double* wq, double* xs, double* buf,
                                              double* Fs, int ld, int warp, int nw) {
  const int lane = threadIdx.x & 31;
  const int l16 = lane & 15, mu = l16 >> 2, nu = l16 & 3, half = lane >> 4;
  const double* __restrict__ ints = m.ints;
  const double* __restrict__ P = m.P;
  const double* __restrict__ H = m.H;
  double* __restrict__ F = m.F;
  const int64_t* __restrict__ row_off = m.row_off;
  const int* __restrict__ first = m.first;
  const int nxx = nh * (nh + 1) / 2;
  // exchange: lane (mu, nu) of half h sums (lam, sig) = ls, ls in [8h, 8h + 8)
  int off[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    const int ls = 8 * half + t;
    off[t] = 10 * pair_index(mu, ls >> 2) + pair_index(nu, ls & 3);
  }
  // Coulomb: lanes 0..9 row r of the block against w_B, lanes 10..19 column q against w_A
  const int cbase = lane < 10 ? 10 * lane : lane - 10, cstep = lane < 10 ? 1 : 10;
  double e = 0.0;
  double pre[4], pv_n = 0.0, h_n = 0.0;
  int A_n = 0, B_n = 0, fA_n = 0, fB_n = 0;
  int a = 0, b = 0;
  if (warp < nxx) tri_inverse(warp, a, b);
  auto fetch = [&]() {
    const int A = hv[a], B = hv[b];
    const double* I = ints + row_off[A] + (int64_t)b * 100 + (int64_t)(B - b) * 10;
#pragma unroll
    for (int k4 = 0; k4 < 4; ++k4) pre[k4] = lane + 32 * k4 < 100 ? I[lane + 32 * k4] : 0.0;
    A_n = A;
    B_n = B;
    fA_n = first[A];
    fB_n = first[B];
    if (A != B) {
      const int64_t ij = tri(fA_n + mu) + fB_n + nu;
      pv_n = P[ij];
      h_n = H[ij];
    }
  };
  if (warp < nxx) fetch();
  for (int k = warp; k < nxx; k += nw) {
#pragma unroll
    for (int k4 = 0; k4 < 4; ++k4)
      if (lane + 32 * k4 < 100) buf[lane + 32 * k4] = pre[k4];
    const int A = A_n, B = B_n, fA = fA_n, fB = fB_n;
    const double pv = pv_n, h = h_n;
    if (k + nw < nxx) {
      b += nw;
      while (b > a) { b -= a + 1; ++a; }
      fetch();
    }
    __syncwarp();
    if (A != B) {
      // G_mu,nu = sum_{lam, sig} P_lam,sig (mu lam | nu sig); lane (lam, sig) holds P_lam,sig
      double g = 0.0;
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const double p = __shfl_sync(0xffffffffu, pv, 8 * half + t);
        g = fma(p, buf[off[t]], g);
      }
      g += __shfl_xor_sync(0xffffffffu, g, 16);
      if (lane < 16) {
        const int i = fA + mu, j = fB + nu;
        const double fv = h - 0.5 * g;
        F[tri(i) + j] = fv;
        if (Fs) {
          Fs[(int64_t)i * ld + j] = fv;
          Fs[(int64_t)j * ld + i] = fv;
        }
        e += pv * (h + fv);
      }
    }
    if (lane < 20) {
      const double* w = wq + wq_offset(m, lane < 10 ? B : A);
      double s = 0.0;
      if (lane < 10 || A != B) {
#pragma unroll
        for (int t = 0; t < 10; ++t) s = fma(buf[cbase + t * cstep], w[t], s);
      }
      xs[(int64_t)k * 20 + lane] = s;
    }
    __syncwarp();
  }
  return e;
}

// Writes F(i, j) = h - g / 2 of an off-diagonal block (h, p preloaded); returns p (h + F).
__device__ __forceinline__ double put_offdiag_h(double* __restrict__ F, double* Fs, int ld, int i,
                                                int j, double p, double g, double h) {
  const double fv = h - 0.5 * g;
  F[tri(i) + j] = fv;
  if (Fs) {
    Fs[(int64_t)i * ld + j] = fv;
    Fs[(int64_t)j * ld + i] = fv;
  }
  return p * (h + fv);
}

// Blocks of atom A with a hydrogen in them: those of its row (B <= A) and of its column
// (rows A2 > A), one block per lane.  Writes A's Coulomb sums over them into J; returns the
// energy share of the row's off-diagonal blocks.  All of a block's loads (integrals, P and H
// entries) are issued before its arithmetic; the restrict-qualified locals let the compiler
// keep them ahead of the previous block's stores.
__device__ __noinline__ double fock_atom_light(const MolView& m, int A, const double* wq,
                                               double* J, double* Fs, int ld) {
  const int lane = threadIdx.x & 31;
  const int na = m.natoms;
  const double* __restrict__ ints = m.ints;
  const double* __restrict__ P = m.P;
  const double* __restrict__ H = m.H;
  double* __restrict__ F = m.F;
  const int8_t* __restrict__ slot = m.slot;
  const int* __restrict__ first = m.first;
  const int* __restrict__ hb = m.hb;
  const int64_t* __restrict__ row_off = m.row_off;
  const int fA = first[A];
  const double* row = ints + row_off[A];
  double e = 0.0;
  if (slot[A] != 0) {
    double jl[10];
#pragma unroll
    for (int r = 0; r < 10; ++r) jl[r] = 0.0;
    // row A, hydrogen B < A: 10 values (pq_A | s_B s_B)
    for (int B = lane; B < A; B += 32) {
      if (slot[B] != 0) continue;
      const int h_ = hb[B], fB = first[B];
      const double* I = row + (int64_t)h_ * 100 + (int64_t)(B - h_) * 10;
      double Iv[10], pl[4], hl[4];
#pragma unroll
      for (int r = 0; r < 10; ++r) Iv[r] = I[r];
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        pl[l] = P[tri(fA + l) + fB];
        hl[l] = H[tri(fA + l) + fB];
      }
      const double w = wq[9 * h_ + B];
#pragma unroll
      for (int r = 0; r < 10; ++r) jl[r] = fma(Iv[r], w, jl[r]);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        double g = 0.0;
#pragma unroll
        for (int l = 0; l < 4; ++l) g = fma(pl[l], Iv[pair_index(u, l)], g);
        e += put_offdiag_h(F, Fs, ld, fA + u, fB, pl[u], g, hl[u]);
      }
    }
    // column A, hydrogen rows A2 > A: 10 values (s_A2 s_A2 | q_A)
    const int hA = hb[A];
    for (int A2 = A + 1 + lane; A2 < na; A2 += 32) {
      if (slot[A2] != 0) continue;
      const double* I = ints + row_off[A2] + (int64_t)hA * 10 + (A - hA);
      const double w = wq[9 * hb[A2] + A2];
#pragma unroll
      for (int r = 0; r < 10; ++r) jl[r] = fma(I[r], w, jl[r]);
    }
    double mine = 0.0;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
      const double v = warp_sum(jl[r]);
      if (lane == r) mine = v;
    }
    if (lane < 10) J[9 * hA + A + lane] = mine;
  } else {
    double jr = 0.0;
    // row A: every B <= A
    for (int B = lane; B <= A; B += 32) {
      const int h_ = hb[B], fB = first[B];
      const double* I = row + (int64_t)h_ * 10 + (B - h_);
      if (slot[B] != 0) {  // 10 values (s_A s_A | q_B)
        double Iv[10], ps[4], hs[4];
#pragma unroll
        for (int q = 0; q < 10; ++q) Iv[q] = I[q];
#pragma unroll
        for (int s_ = 0; s_ < 4; ++s_) {
          ps[s_] = P[tri(fA) + fB + s_];
          hs[s_] = H[tri(fA) + fB + s_];
        }
        const double* wB = wq + 9 * h_ + B;
#pragma unroll
        for (int q = 0; q < 10; ++q) jr = fma(Iv[q], wB[q], jr);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          double g = 0.0;
#pragma unroll
          for (int s_ = 0; s_ < 4; ++s_) g = fma(ps[s_], Iv[pair_index(v, s_)], g);
          e += put_offdiag_h(F, Fs, ld, fA, fB + v, ps[v], g, hs[v]);
        }
      } else {
        const double I0 = I[0];
        jr = fma(I0, wq[9 * h_ + B], jr);
        if (B < A) {
          const int64_t ij = tri(fA) + fB;
          const double p = P[ij], h = H[ij];
          e += put_offdiag_h(F, Fs, ld, fA, fB, p, p * I0, h);
        }
      }
    }
    // column A: every row A2 > A
    const int hA = hb[A];
    for (int A2 = A + 1 + lane; A2 < na; A2 += 32) {
      const bool h2 = slot[A2] != 0;
      const double* I = ints + row_off[A2] + (h2 ? (int64_t)hA * 100 + (int64_t)(A - hA) * 10
                                                 : (int64_t)hA * 10 + (A - hA));
      const double* w2 = wq + 9 * hb[A2] + A2;
      if (h2) {
        double s_ = 0.0;
#pragma unroll
        for (int r = 0; r < 10; ++r) s_ = fma(I[r], w2[r], s_);
        jr += s_;
      } else {
        jr = fma(I[0], w2[0], jr);
      }
    }
    jr = warp_sum(jr);
    if (lane == 0) J[9 * hA + A] = jr;
  }
  return e;
}

// Diagonal block element (A, pq): H + J - 1/2 one-center exchange; its share of E_el.  The
// atom's P block and the heavy-heavy partial sums are read before the arithmetic.
__device__ __forceinline__ double fock_diag_final(const MolView& m, const double* J,
                                                  const double* xs, int nh, double* Fs, int ld,
                                                  int t) {
  const int A = t / 10, pq = t % 10;
  const int sA = m.slot[A];
  if (sA == 0 && pq) return 0.0;
  const int a = pair_first(pq), b = pair_second(pq), fA = m.first[A];
  const int nA = nao_of_slot(sA);
  double Pa[16];
#pragma unroll
  for (int l = 0; l < 4; ++l)
#pragma unroll
    for (int s = 0; s < 4; ++s) Pa[4 * l + s] = (l < nA && s < nA) ? m.P[pk(fA + l, fA + s)] : 0.0;
  double Jv = J[wq_offset(m, A) + pq];
  if (sA != 0) {  // heavy-heavy partial sums: rows b <= a, then columns b > a
    const int a_ = m.hb[A];
    double r0 = 0.0, r1 = 0.0;
    for (int b_ = 0; b_ <= a_; ++b_) r0 += xs[(tri(a_) + b_) * 20 + pq];
    for (int b_ = a_ + 1; b_ < nh; ++b_) r1 += xs[(tri(b_) + a_) * 20 + 10 + pq];
    Jv += r0 + r1;
  }
  double K = 0.0;
#pragma unroll
  for (int l = 0; l < 4; ++l)
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      if (l >= nA || s >= nA) continue;
      const double x = one_center_value(sA, a < l ? a : l, a < l ? l : a, b < s ? b : s, b < s ? s : b);
      if (x != 0.0) K += Pa[4 * l + s] * x;
    }
  const int i = fA + b, j = fA + a;  // i >= j
  const int64_t ij = tri(i) + j;
  const double h = m.H[ij], fv = h + (Jv - 0.5 * K);
  m.F[ij] = fv;
  if (Fs) {
    Fs[(int64_t)i * ld + j] = fv;
    Fs[(int64_t)j * ld + i] = fv;
  }
  return m.P[ij] * (h + fv) * (i == j ? 0.5 : 1.0);
}

// F (packed, and full into Fs when given, row stride ld) and E_el for the density in m.P.
// wq, J: 10 n_heavy + n_light doubles each; stage: kFockStage doubles; hv: n_heavy ints (all
// shared memory); xs: fock_xx_doubles(nao) doubles (shared or global memory).
template <int NT>
__device__ double block_fock_energy(const MolView& m, double* Fs, int ld, double* wq, double* J,
                                    double* stage, double* xs, int* hv, double* red) {
  constexpr int NW = NT / 32;
  const int warp = threadIdx.x >> 5;
  const int na = m.natoms;
  for (int t = threadIdx.x; t < na * 10; t += NT) pair_density_task(m, wq, t);
  for (int A = threadIdx.x; A < na; A += NT)
    if (m.slot[A] != 0) hv[m.hb[A]] = A;
  const int nh = m.hb[na - 1] + (m.slot[na - 1] != 0);
  __syncthreads();
  double e = fock_xx_blocks(m, hv, nh, wq, xs, stage + warp * kFockStagePerWarp, Fs, ld, warp, NW);
  for (int A = warp; A < na; A += NW) e += fock_atom_light(m, A, wq, J, Fs, ld);
  __syncthreads();
  for (int t = threadIdx.x; t < na * 10; t += NT) e += fock_diag_final(m, J, xs, nh, Fs, ld, t);
  return block_sum<NT>(e, red);
}

}  // namespace sgb
