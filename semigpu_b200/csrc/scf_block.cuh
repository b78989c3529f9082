// CTA-cooperative stages of one molecule's MNDO calculation.  Every function here is called by
// all threads of one thread block and works on one molecule (a MolView); the persistent batch
// kernel strings them together so a molecule's whole SCF runs inside one CTA with its Fock /
// Jacobi matrix resident in shared memory.
//
// Reference stages (LuisAlfredoNu/semiGPU, src/common):
//   integrals  ComputeAllTwoCenterIntegral      twocenterintegral.cpp:229-279
//   Hcore      Hcore::ComputeElementMatrix      hcore.cpp:25-100
//   guess      DensityMatrix guess              densitymatrix.cpp:26-37
//   Fock       FockMatrix / ComputeGMatrix_UV   fockmatrix.cpp:20-53, twoelectronmatrix.cpp:14-35
//   energy     ElectronicEnergy::ComputeEnergy  electronicenergy.cpp:12-36
//   eigensolve GetEigenValVecOfFmatrix (dsyev)  scfcalculation.cpp:171-203
//   density    DensityMatrix::ComputeElementMatrix densitymatrix.cpp:38-46
//   core-core  CoreCoreRepulsion                corecorerepulsion.cpp:12-65
//
// The Fock build uses the NDDO sparsity of the reference's own sum: (mu nu|lam sig) is zero
// unless mu, nu share an atom and lam, sig share an atom (GetValueFromArray,
// twocenterintegral.cpp:285-386), so F = H + G(P) reduces to a Coulomb sum per atom over all
// atoms, a one-center exchange per atom and a two-center exchange per atom pair.
#pragma once
#include "layout.h"
#include "mndo_device.cuh"

namespace sgb {

struct MolView {
  int natoms, nao, nocc;
  const int8_t* slot;      // per atom
  const double* pos;       // 3 per atom, bohr
  const int* first;        // first AO of each atom
  const int64_t* row_off;  // integral block-row offsets
  const int* hb;           // heavy atoms before each atom
  double* ints;            // integral blocks
  double* H;               // packed
  double* P;               // packed
  double* F;               // packed
  double* V;               // n*n, row-major: V[i*n + k] = AO i of vector k
  double* T;               // n*n scratch
  double* eig;             // n
  double* W;               // n*n eigensolver work matrix in global memory (large molecules)
};

__device__ __forceinline__ int nao_of_slot(int s) { return s ? 4 : 1; }

__device__ __forceinline__ const double* blk_ptr(const MolView& m, int A, int B) {
  return m.ints + block_offset(m.row_off, m.hb, m.slot, A, B);
}

// atom pair index p -> (A, B) with A >= B, p = A(A+1)/2 + B
__device__ __forceinline__ void tri_inverse(int64_t p, int& A, int& B) {
  int a = (int)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
  while (tri(a + 1) <= p) ++a;
  while (tri(a) > p) --a;
  A = a;
  B = (int)(p - tri(a));
}

// Block-wide sum (all threads call; result valid in every thread).
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (l < NT / 32) ? red[l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (l == 0) red[0] = v;
  }
  __syncthreads();
  double r = red[0];
  __syncthreads();
  return r;
}

// ------------------------------------------------------------------------------------------
// Integrals: one thread per atom pair (A >= B), writing the pair's block.
__device__ __noinline__ void write_pair_block(const MolView& m, int A, int B) {
  double* blk = m.ints + block_offset(m.row_off, m.hb, m.slot, A, B);
  const int sA = m.slot[A], sB = m.slot[B];
  if (A == B) {
    if (sA == 0) {
      blk[0] = c_elem[0].gss;
    } else {
      for (int i = 0; i < 10; ++i)
        for (int j = 0; j < 10; ++j)
          blk[10 * i + j] = one_center_value(sA, pair_first(i), pair_second(i), pair_first(j),
                                             pair_second(j));
    }
    return;
  }
  PairFrame f;
  if (sA != 0 && sB != 0) {
    pair_frame(sA, sB, m.pos + 3 * A, m.pos + 3 * B, f);
    for (int i = 0; i < 10; ++i) {
      const int a = pair_first(i), b = pair_second(i);
      for (int j = 0; j < 10; ++j)
        blk[10 * i + j] = two_center_value(f, a, b, pair_first(j), pair_second(j));
    }
  } else if (sA == 0 && sB == 0) {
    pair_frame(0, 0, m.pos + 3 * A, m.pos + 3 * B, f);
    blk[0] = f.v[L_SSSS] * kHartree2eV;
  } else {
    // H-X and X-H blocks hold (s_H s_H | pair on X), computed with the H atom first
    // (ComputePair_HX / ComputePair_XH, twocenterintegral.cpp:400-447).
    const int Hh = sA == 0 ? A : B, X = sA == 0 ? B : A;
    pair_frame(0, m.slot[X], m.pos + 3 * Hh, m.pos + 3 * X, f);
    for (int k = 0; k < 10; ++k) blk[k] = two_center_value(f, 0, 0, pair_first(k), pair_second(k));
  }
}

__device__ inline void block_integrals(const MolView& m) {
  const int64_t np = tri(m.natoms);
  for (int64_t p = threadIdx.x; p < np; p += blockDim.x) {
    int A, B;
    tri_inverse(p, A, B);
    write_pair_block(m, A, B);
  }
}

// (mu nu | s_C s_C) for mu, nu on atom A (pair index pq of A), C != A.
__device__ __forceinline__ double coulomb_ss(const MolView& m, int A, int pq, int C) {
  const int sA = m.slot[A], sC = m.slot[C];
  if (sA == 0) return *blk_ptr(m, A > C ? A : C, A > C ? C : A);   // (sA sA|sC sC): entry 0
  if (sC == 0) return blk_ptr(m, A > C ? A : C, A > C ? C : A)[pq];  // H-X block, column pq
  return A > C ? blk_ptr(m, A, C)[10 * pq] : blk_ptr(m, C, A)[pq];
}

// Hcore: off-diagonal atom blocks 1/2 (beta_mu + beta_nu) S_mu_nu (hcore.cpp:38-69), diagonal
// atom blocks U delta + sum_{C != A} -Z_C (mu nu|s_C s_C) (hcore.cpp:71-92).
__device__ __noinline__ void hcore_offdiag_pair(const MolView& m, int A, int B) {
  const int sA = m.slot[A], sB = m.slot[B];
  double S[16];
  overlap_block(sA, sB, m.pos + 3 * A, m.pos + 3 * B, S);
  const int nA = nao_of_slot(sA), nB = nao_of_slot(sB), fA = m.first[A], fB = m.first[B];
  for (int mu = 0; mu < nA; ++mu) {
    const double ba = mu ? c_elem[sA].beta_p : c_elem[sA].beta_s;
    for (int nu = 0; nu < nB; ++nu) {
      const double bb = nu ? c_elem[sB].beta_p : c_elem[sB].beta_s;
      m.H[tri(fA + mu) + fB + nu] = (ba + bb) * S[4 * mu + nu] * 0.5;
    }
  }
}

__device__ __noinline__ void hcore_diag_atom(const MolView& m, int A, int pq) {
  const int sA = m.slot[A];
  double s = 0.0;
  for (int C = 0; C < m.natoms; ++C)
    if (C != A) s += -(double)c_elem[m.slot[C]].core * coulomb_ss(m, A, pq, C);
  const int a = pair_first(pq), b = pair_second(pq), f = m.first[A];
  if (a == b) s += a == 0 ? c_elem[sA].uss : c_elem[sA].upp;
  m.H[tri(f + b) + f + a] = s;
}

__device__ inline void block_hcore(const MolView& m) {
  const int64_t np = tri(m.natoms);
  // diagonal blocks first: one task per (atom, pair index)
  for (int t = threadIdx.x; t < m.natoms * 10; t += blockDim.x) {
    const int A = t / 10, pq = t % 10;
    if (m.slot[A] == 0 && pq) continue;
    hcore_diag_atom(m, A, pq);
  }
  for (int64_t p = threadIdx.x; p < np; p += blockDim.x) {
    int A, B;
    tri_inverse(p, A, B);
    if (A != B) hcore_offdiag_pair(m, A, B);
  }
}

// ------------------------------------------------------------------------------------------
// Fock build + electronic energy.  Writes F packed to global memory and, when Fs != nullptr,
// the full symmetric F (leading dimension ld).
//
// wq: scratch of 10 * nheavy + nlight doubles: the pair densities of each atom,
//     w_C[q] = P_{lam sig} (x2 when lam != sig) for pair q = (lam, sig) of atom C.
__device__ __forceinline__ int wq_offset(const MolView& m, int A) { return 9 * m.hb[A] + A; }

// Per-task pieces of the grid-wide kernels (the one-CTA build is in fock_block.cuh).

// w_C[q] for task t = (C, q)
__device__ __forceinline__ void pair_density_task(const MolView& m, double* wq, int t) {
  const int C = t / 10, q = t % 10;
  const int s = m.slot[C];
  if (s == 0 && q) return;
  const int a = pair_first(q), b = pair_second(q), f = m.first[C];
  const double p = m.P[tri(f + b) + f + a];
  wq[wq_offset(m, C) + q] = a == b ? p : 2.0 * p;
}

// Diagonal atom block element (A, pq): Coulomb over every atom plus one-center exchange.
// Returns the element's share of E_el.
__device__ __noinline__ double fock_diag_task(const MolView& m, const double* wq, double* Fs,
                                        int64_t ld, int t) {
  const int A = t / 10, pq = t % 10;
  const int sA = m.slot[A];
  if (sA == 0 && pq) return 0.0;
  const int a = pair_first(pq), b = pair_second(pq), fA = m.first[A];
  double J = 0.0;
  for (int C = 0; C < m.natoms; ++C) {
    const int sC = m.slot[C];
    const double* w = wq + wq_offset(m, C);
    if (sA == 0) {
      if (sC == 0) {
        J += *blk_ptr(m, A > C ? A : C, A > C ? C : A) * w[0];
      } else {
        const double* I = blk_ptr(m, A > C ? A : C, A > C ? C : A);
#pragma unroll
        for (int q = 0; q < 10; ++q) J += I[q] * w[q];
      }
    } else if (sC == 0) {
      J += blk_ptr(m, A > C ? A : C, A > C ? C : A)[pq] * w[0];
    } else if (A >= C) {
      const double* I = blk_ptr(m, A, C) + 10 * pq;
#pragma unroll
      for (int q = 0; q < 10; ++q) J += I[q] * w[q];
    } else {
      const double* I = blk_ptr(m, C, A) + pq;
#pragma unroll
      for (int q = 0; q < 10; ++q) J += I[10 * q] * w[q];
    }
  }
  // one-center exchange -1/2 sum_{lam,sig in A} P_lam_sig (mu lam|nu sig)
  double K = 0.0;
  const int nA = nao_of_slot(sA);
  for (int l = 0; l < nA; ++l)
    for (int s = 0; s < nA; ++s) {
      const double x = one_center_value(sA, a < l ? a : l, a < l ? l : a, b < s ? b : s, b < s ? s : b);
      if (x != 0.0) K += m.P[pk(fA + l, fA + s)] * x;
    }
  const int i = fA + b, j = fA + a;  // i >= j
  const int64_t ij = tri(i) + j;
  const double h = m.H[ij], fv = h + (J - 0.5 * K);
  m.F[ij] = fv;
  if (Fs) { Fs[i * ld + j] = fv; Fs[j * ld + i] = fv; }
  return m.P[ij] * (h + fv) * (i == j ? 0.5 : 1.0);
}

// Off-diagonal atom block (A > B): two-center exchange only.  Returns its share of E_el.
__device__ __noinline__ double fock_pair_task(const MolView& m, double* Fs, int64_t ld, int A, int B) {
  const int sA = m.slot[A], sB = m.slot[B], fA = m.first[A], fB = m.first[B];
  const double* I = blk_ptr(m, A, B);
  const int nA = nao_of_slot(sA), nB = nao_of_slot(sB);
  double Pab[16];
  for (int l = 0; l < nA; ++l)
    for (int s = 0; s < nB; ++s) Pab[4 * l + s] = m.P[tri(fA + l) + fB + s];
  double e = 0.0;
  for (int mu = 0; mu < nA; ++mu)
    for (int nu = 0; nu < nB; ++nu) {
      double g = 0.0;
      if (sA != 0 && sB != 0) {
        for (int l = 0; l < 4; ++l) {
          const double* Ir = I + 10 * pair_index(mu, l);
#pragma unroll
          for (int s = 0; s < 4; ++s) g += Pab[4 * l + s] * Ir[pair_index(nu, s)];
        }
      } else if (sA != 0) {  // B is H: (mu lam | s_B s_B), block column = pair(mu, lam)
        for (int l = 0; l < 4; ++l) g += Pab[4 * l] * I[pair_index(mu, l)];
      } else if (sB != 0) {  // A is H: (s_A s_A | nu sig)
        for (int s = 0; s < 4; ++s) g += Pab[s] * I[pair_index(nu, s)];
      } else {
        g = Pab[0] * I[0];
      }
      const int i = fA + mu, j = fB + nu;
      const int64_t ij = tri(i) + j;
      const double h = m.H[ij], fv = h - 0.5 * g;
      m.F[ij] = fv;
      if (Fs) { Fs[i * ld + j] = fv; Fs[j * ld + i] = fv; }
      e += m.P[ij] * (h + fv);
    }
  return e;
}

// Initial guess P_ii = Z_A / nAO_A, zero elsewhere (densitymatrix.cpp:26-37).
__device__ inline void block_guess(const MolView& m) {
  const int64_t np = tri(m.nao);
  for (int64_t t = threadIdx.x; t < np; t += blockDim.x) m.P[t] = 0.0;
  __syncthreads();
  for (int A = threadIdx.x; A < m.natoms; A += blockDim.x) {
    const int s = m.slot[A], n = nao_of_slot(s), f = m.first[A];
    for (int k = 0; k < n; ++k) m.P[tri(f + k) + f + k] = (double)c_elem[s].core / n;
  }
}

// Core-core repulsion of atoms Al < Bh (corecorerepulsion.cpp:12-65):
// Z_A Z_B (s_A s_A|s_B s_B) f(R), R in Angstrom; N-H / O-H use 1 + R exp(-alpha_X R) + exp(-alpha_H R).
__device__ __noinline__ double core_core_pair(const MolView& m, int Bh, int Al) {
  const int sa = m.slot[Al], sb = m.slot[Bh];
  const double gam = *blk_ptr(m, Bh, Al);
  const double* pa = m.pos + 3 * Al;
  const double* pb = m.pos + 3 * Bh;
  const double dx = pa[0] - pb[0], dy = pa[1] - pb[1], dz = pa[2] - pb[2];
  const double r = sqrt(dx * dx + dy * dy + dz * dz) * kBohr2Ang;
  const int za = c_elem[sa].z, zb = c_elem[sb].z;
  double f;
  if (zb == 1 && (za == 7 || za == 8))
    f = 1.0 + r * exp(-c_elem[sa].alpha * r) + exp(-c_elem[sb].alpha * r);
  else if (za == 1 && (zb == 7 || zb == 8))
    f = 1.0 + r * exp(-c_elem[sb].alpha * r) + exp(-c_elem[sa].alpha * r);
  else
    f = 1.0 + exp(-c_elem[sa].alpha * r) + exp(-c_elem[sb].alpha * r);
  return (double)(c_elem[sa].core * c_elem[sb].core) * gam * f;
}

template <int NT>
__device__ double block_core_core(const MolView& m, double* red) {
  double e = 0.0;
  const int64_t np = tri(m.natoms);
  for (int64_t p = threadIdx.x; p < np; p += blockDim.x) {
    int Bh, Al;
    tri_inverse(p, Bh, Al);
    if (Bh != Al) e += core_core_pair(m, Bh, Al);
  }
  return block_sum<NT>(e, red);
}

// ------------------------------------------------------------------------------------------
// Dense helpers on one CTA.

template <int NT>
__device__ __forceinline__ double block_max(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (l < NT / 32) ? red[l] : -INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (l == 0) red[0] = v;
  }
  __syncthreads();
  double r = red[0];
  __syncthreads();
  return r;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Warp sums of four values, every lane receiving all four.  The first two butterfly levels
// split the values between lane halves (each lane forwards the sums it does not keep), so the
// reduction costs 6 exchanges plus 4 broadcasts instead of 4 x 5 exchanges.
__device__ __forceinline__ void warp_sum4(int lane, double& a, double& b, double& c, double& d) {
  const bool hi16 = lane & 16, hi8 = lane & 8;
  // level 16: lower half keeps (a, b), upper half keeps (c, d)
  double x = __shfl_xor_sync(0xffffffffu, hi16 ? a : c, 16);
  double y = __shfl_xor_sync(0xffffffffu, hi16 ? b : d, 16);
  double k0 = (hi16 ? c : a) + x;
  double k1 = (hi16 ? d : b) + y;
  // level 8: lanes with bit 3 clear keep k0, set keep k1
  const double z = __shfl_xor_sync(0xffffffffu, hi8 ? k0 : k1, 8);
  double v = (hi8 ? k1 : k0) + z;
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  // lane 0 holds a, lane 8 b, lane 16 c, lane 24 d
  a = __shfl_sync(0xffffffffu, v, 0);
  b = __shfl_sync(0xffffffffu, v, 8);
  c = __shfl_sync(0xffffffffu, v, 16);
  d = __shfl_sync(0xffffffffu, v, 24);
}

// Shift making F + mu I positive semi-definite: mu = ||F||_inf + 1 (row sums of |F_ij|).
template <int NT>
__device__ double block_shift(int n, const double* Ffull, double* red) {
  double mx = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double s = 0.0;
    const double* row = Ffull + (int64_t)i * n;
    for (int j = 0; j < n; ++j) s += fabs(row[j]);
    mx = fmax(mx, s);
  }
  return block_max<NT>(mx, red) + 1.0;
}

// G (column-major, ldg) = (F + mu I) V with F full symmetric (row-major = column-major, n x n,
// ld n) and V column-major (ldv); 4x4 register tiles.
__device__ inline void block_shifted_product(int n, const double* F, double mu, const double* V,
                                             int ldv, double* G, int ldg) {
  const int tiles = (n + 3) >> 2;
  for (int t = threadIdx.x; t < tiles * tiles; t += blockDim.x) {
    const int i0 = (t % tiles) * 4, j0 = (t / tiles) * 4;
    double acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
    const double* fr[4];
    const double* vc[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) fr[r] = F + (int64_t)(i0 + r < n ? i0 + r : n - 1) * n;
#pragma unroll
    for (int c = 0; c < 4; ++c) vc[c] = V + (int64_t)(j0 + c < n ? j0 + c : n - 1) * ldv;
    for (int l = 0; l < n; ++l) {
      double a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = fr[r][l];
#pragma unroll
      for (int c = 0; c < 4; ++c) b[c] = vc[c][l];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int i = i0 + r, j = j0 + c;
        if (i < n && j < n) G[(int64_t)j * ldg + i] = fma(mu, vc[c][i], acc[r][c]);
      }
  }
}

// ------------------------------------------------------------------------------------------
// Cyclic Jacobi on A = V^T F V carried out on columns only.  The CTA keeps V (orthogonal,
// column-major) and G = F V; a two-sided rotation J of A in the (p, q) plane is
// A <- J^T A J, which is exactly V <- V J together with G <- G J.  Its angle needs
// A_pp = v_p.g_p, A_qq = v_q.g_q and A_pq = (v_p.g_q + g_p.v_q) / 2 -- four dot products of the
// pair's own columns -- so one warp owns one column pair per round (columns in registers,
// n <= 32 * CR) and a round needs one barrier.  Convergence is that of two-sided Jacobi on
// F (no spectral shift).  Pairs follow the round-robin ordering (ne = n rounded up to even,
// m = ne - 1: round r pairs m with r and (r + k) % m with (r - k) % m; an index >= n is a
// dummy).  CR doubles per lane hold one column, so n <= 32 * CR.
//
// The rotation's tangent is computed in FP32 (an approximate angle only leaves a residual the
// next sweep removes); c = rsqrt(1 + t^2) and s = c t are FP64, so every applied rotation is
// orthogonal to rounding.  A pair is skipped when |A_pq| <= rot_abs; sweeps stop after one
// whose largest |A_pq| was below done_abs (the next would start from about its square over the
// gap).  Returns the sweep count, or -1 (max_sweeps exhausted or a non-finite value).
__device__ __forceinline__ void rr_pair(int r, int k, int m, int& p, int& q) {
  if (k == 0) { p = m; q = r; }
  else {
    p = r + k; if (p >= m) p -= m;
    q = r - k; if (q < 0) q += m;
  }
}

//
// Bipartite mode (grp_a != nullptr): only pairs between the index sets grp_a (na entries) and
// grp_b (nb entries, na <= nb) are rotated -- round r pairs grp_a[k] with grp_b[(k + r) % nb],
// nb rounds per sweep.  The SCF uses it with the occupied and virtual columns: the density
// matrix only depends on the occupied subspace, which these rotations alone decide.
// Each warp carries PP column pairs of a round at once (independent dependency chains
// interleaved), which hides the latency of the dot-product reduction and the angle computation.
// CR == 0: columns too long for registers (nao > 160, G and V in global memory); each pair is
// streamed twice, once for the dot products and once for the rotation.
template <int NT>
__device__ void jacobi_pair_streamed(int n, double* gp, double* gq, double* vp, double* vq,
                                     int lane, double rot_abs, double& worst) {
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
  if (!(fabs(a_pq) > rot_abs)) {
    if (a_pq != a_pq) worst = INFINITY;
    return;
  }
  worst = fmax(worst, fabs(a_pq));
  const float num = (float)(2.0 * a_pq), den = (float)(aqq - app);
  float tf = __fdividef(num, fabsf(den) + __fsqrt_rn(fmaf(den, den, num * num)));
  if (den < 0.0f) tf = -tf;
  const double t = (double)tf;
  const double c = rsqrt(fma(t, t, 1.0)), sn = c * t;
  for (int i = lane; i < n; i += 32) {
    const double xg = gp[i], yg = gq[i], xv = vp[i], yv = vq[i];
    gp[i] = c * xg - sn * yg;
    gq[i] = sn * xg + c * yg;
    vp[i] = c * xv - sn * yv;
    vq[i] = sn * xv + c * yv;
  }
}

template <int NT, int CR, int PP = 2>
__device__ int block_jacobi_fv(int n, double* G, int ldg, double* V, int ldv, double* red,
                               double rot_abs, double done_abs, int max_sweeps,
                               const int* grp_a = nullptr, int na = 0, const int* grp_b = nullptr,
                               int nb = 0) {
  if constexpr (CR == 0) {
    const int ne = n + (n & 1), m = ne - 1, n2 = ne / 2;
    const bool bip = grp_a != nullptr;
    const int rounds = bip ? nb : m, per_round = bip ? na : n2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int sweep = 0; sweep < max_sweeps; ++sweep) {
      double worst = 0.0;
      for (int r = 0; r < rounds; ++r) {
        for (int k = warp; k < per_round; k += NT / 32) {
          int p, q;
          if (bip) {
            p = grp_a[k];
            int j = k + r;
            if (j >= nb) j -= nb;
            q = grp_b[j];
          } else {
            rr_pair(r, k, m, p, q);
            if (p >= n || q >= n) continue;
          }
          jacobi_pair_streamed<NT>(n, G + (int64_t)p * ldg, G + (int64_t)q * ldg,
                                   V + (int64_t)p * ldv, V + (int64_t)q * ldv, lane, rot_abs,
                                   worst);
        }
        __syncthreads();
      }
      worst = block_max<NT>(worst, red);
      if (!(worst < INFINITY)) return -1;
      if (worst < done_abs) return sweep + 1;
    }
    return -1;
  } else {
  const int ne = n + (n & 1), m = ne - 1, n2 = ne / 2;
  const bool bip = grp_a != nullptr;
  const int rounds = bip ? nb : m, per_round = bip ? na : n2;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int NW = NT / 32;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    double worst = 0.0;
    for (int r = 0; r < rounds; ++r) {
      for (int k0 = warp; k0 < per_round; k0 += PP * NW) {
        int p[PP], q[PP];
        bool live[PP];
#pragma unroll
        for (int u = 0; u < PP; ++u) {
          const int k = k0 + u * NW;
          live[u] = k < per_round;
          p[u] = 0;
          q[u] = 0;
          if (live[u]) {
            if (bip) {
              p[u] = grp_a[k];
              int j = k + r;
              if (j >= nb) j -= nb;
              q[u] = grp_b[j];
            } else {
              rr_pair(r, k, m, p[u], q[u]);
              live[u] = p[u] < n && q[u] < n;
              if (!live[u]) p[u] = q[u] = 0;
            }
          }
        }
        double xg[PP][CR], yg[PP][CR], xv[PP][CR], yv[PP][CR];
        double app[PP], aqq[PP], apq[PP], aqp[PP];
#pragma unroll
        for (int u = 0; u < PP; ++u) {
          const double* gp = G + (int64_t)p[u] * ldg;
          const double* gq = G + (int64_t)q[u] * ldg;
          const double* vp = V + (int64_t)p[u] * ldv;
          const double* vq = V + (int64_t)q[u] * ldv;
#pragma unroll
          for (int j = 0; j < CR; ++j) {
            const int i = lane + 32 * j;
            const bool in = live[u] && i < n;
            xg[u][j] = in ? gp[i] : 0.0;
            yg[u][j] = in ? gq[i] : 0.0;
            xv[u][j] = in ? vp[i] : 0.0;
            yv[u][j] = in ? vq[i] : 0.0;
          }
        }
#pragma unroll
        for (int u = 0; u < PP; ++u) {
          app[u] = aqq[u] = apq[u] = aqp[u] = 0.0;
#pragma unroll
          for (int j = 0; j < CR; ++j) {
            app[u] = fma(xv[u][j], xg[u][j], app[u]);
            aqq[u] = fma(yv[u][j], yg[u][j], aqq[u]);
            apq[u] = fma(xv[u][j], yg[u][j], apq[u]);
            aqp[u] = fma(xg[u][j], yv[u][j], aqp[u]);
          }
        }
#pragma unroll
        for (int u = 0; u < PP; ++u) warp_sum4(lane, app[u], aqq[u], apq[u], aqp[u]);
#pragma unroll
        for (int u = 0; u < PP; ++u) {
          const double a_pq = 0.5 * (apq[u] + aqp[u]);
          if (!live[u]) continue;
          if (!(fabs(a_pq) > rot_abs)) {
            if (a_pq != a_pq) worst = INFINITY;
            continue;
          }
          worst = fmax(worst, fabs(a_pq));
          // tan of the angle zeroing A_pq: t = sgn(den) num / (|den| + hypot(den, num)),
          // num = 2 A_pq, den = A_qq - A_pp (the smaller of the two roots)
          // approximate FP32 arithmetic is enough here: the angle may be slightly off, the
          // rotation applied below is exactly orthogonal
          const float num = (float)(2.0 * a_pq), den = (float)(aqq[u] - app[u]);
          float tf = __fdividef(num, fabsf(den) + __fsqrt_rn(fmaf(den, den, num * num)));
          if (den < 0.0f) tf = -tf;
          const double t = (double)tf;
          const double c = rsqrt(fma(t, t, 1.0)), sn = c * t;
          double* gp = G + (int64_t)p[u] * ldg;
          double* gq = G + (int64_t)q[u] * ldg;
          double* vp = V + (int64_t)p[u] * ldv;
          double* vq = V + (int64_t)q[u] * ldv;
#pragma unroll
          for (int j = 0; j < CR; ++j) {
            const int i = lane + 32 * j;
            if (i < n) {
              gp[i] = c * xg[u][j] - sn * yg[u][j];
              gq[i] = sn * xg[u][j] + c * yg[u][j];
              vp[i] = c * xv[u][j] - sn * yv[u][j];
              vq[i] = sn * xv[u][j] + c * yv[u][j];
            }
          }
        }
      }
      __syncthreads();
    }
    worst = block_max<NT>(worst, red);
    if (!(worst < INFINITY)) return -1;
    if (worst < done_abs) return sweep + 1;
  }
  return -1;
  }
}

// eig[i] = g_i . v_i - mu (one warp per column)
template <int NT>
__device__ void block_rayleigh(int n, const double* G, int ldg, const double* V, int ldv,
                               double mu, double* eig) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = warp; i < n; i += NT / 32) {
    double s = 0.0;
    for (int k = lane; k < n; k += 32) s = fma(G[(int64_t)i * ldg + k], V[(int64_t)i * ldv + k], s);
    s = warp_sum(s);
    if (lane == 0) eig[i] = s - mu;
  }
}

}  // namespace sgb
