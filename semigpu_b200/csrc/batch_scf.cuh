// Persistent batched SCF: one CTA runs one molecule's whole calculation (integrals, Hcore,
// guess, SCF loop, core-core repulsion) and then takes the next molecule from a work counter.
// Molecules are handed out in the order given by `order` (the host sorts by estimated cost,
// largest first, so the tail of the launch holds the cheap ones).
//
// Shared memory holds the matrix the density step works on (purification's X, or the Jacobi
// working matrix G = F V and, for nao <= 110, the eigenvectors V), which the Fock build reuses
// as staging space; the per-atom pair densities, Coulomb sums and a few reduction slots follow.
// Hcore, P, F (packed and full) live in global memory (L2-resident at these sizes), as do V and,
// above nao 160, the work matrices.
//
// The SCF loop is the reference's (scfcalculation.cpp:66-146): guess P -> F -> E_0, then
// repeat {eigensolve F -> P from the nocc lowest vectors -> F -> E} until |dE| < tol or
// max_iter steps.  Two ways to get P from F, chosen per launch:
//  * SOLVER_PURIFY (default): P by trace-correcting purification, ~20 symmetric matrix
//    squares on the FP64 tensor-core path (purify.cuh; X in shared memory up to nao 160, in
//    global memory above); a Jacobi eigensolve replaces it for a step whose purification fails
//    (vanishing gap), and runs once at the end when the eigenpairs are wanted (single-molecule
//    calls).
//  * SOLVER_JACOBI: a cyclic Jacobi on V^T F V carried on the columns of V and G = F V; after
//    the first step it is warm-started from the previous eigenvectors, which the new F barely
//    mixes, so it needs few sweeps.
#pragma once
#include "dmma_tiles.cuh"
#include "fock_block.cuh"
#include "tf32_tiles.cuh"
#include "purify.cuh"
#include "scf_block.cuh"

namespace sgb {

constexpr int kBatchJacobiSweeps = 40;
constexpr int kWorkMaps = 6;  // tensor maps per molecule above nao 160

struct BatchArgs {
  int nmol;
  const MolDesc* mols;
  const int* order;
  int* counter;
  const int8_t* slot;
  const double* pos;
  const int* first;
  const int64_t* row_off;
  const int* hb;
  double* ints;
  double* H;
  double* P;
  double* F;
  double* V;
  double* T;
  double* eig;
  double* W;        // work matrices (X and its partner, or G) of the molecules above nao 160
  // tensor maps of the work matrices of the molecules above nao 160, kWorkMaps per molecule:
  // X and its partner as FP64, then the TF32 hi / lo parts of the two sets of the mixed form
  const CUtensorMap* wmaps = nullptr;
  double* e_el;
  double* e_cc;
  int* n_iter;
  int* converged;
  int* status;
  double* hist;     // optional energy history, hist_stride doubles per molecule
  int hist_stride;
  double tol;
  int max_iter;
  int nmax;         // largest nao in the launch (sizes the shared memory)
  size_t mat_doubles;  // shared matrix region (max over molecules of mat_doubles_for)
  int sorted_vectors;  // eigenvalues and sorted eigenvectors of the last eigensolve wanted
  int solver;       // SOLVER_*
  int stages;       // STAGE_* bits
  unsigned long long* t_begin;  // optional per-molecule %globaltimer (ns) at start / end
  unsigned long long* t_end;
  unsigned long long* stage_cycles;  // optional, kStageSlots SM cycles per molecule
  // Pulay DIIS (launched only with it on): (2 depth + 1) n^2 doubles of history per molecule
  // at (2 depth + 1) sq0, and kDiisB doubles of B matrix per molecule
  double* diis = nullptr;
  double* diis_B = nullptr;
  int diis_depth = 0;
  // Limits of the bounded loops: Jacobi sweeps per eigensolve (a non-converged eigensolve
  // stops the molecule's SCF with MOL_EIG_FAILED, the reference's LAPACK info > 0 break), and
  // polls of the first wait for a product's tensor-core MMAs (a timed-out wait abandons the
  // purification of that step, which is then diagonalised).
  int max_sweeps = kBatchJacobiSweeps;
  long long wait_spins = kMbarSpins;
  // Density damping (0 = off, the reference's plain loop): each step's density is mixed with
  // the previous one, P = (1 - damping) P_new + damping P_old, before the Fock build.
  double damping = 0.0;
};

// Stage timers (SM clock cycles of the CTA, thread 0, between block-wide barriers), the
// analogue of the reference's per-step Lapack/Pmat/Fmat/Ener timers
// (scfcalculation.cpp:83-140).
enum : int { ST_INTS = 0, ST_HCORE, ST_FOCK, ST_SHIFT_GEMM, ST_JACOBI, ST_EIGVAL_SORT,
             ST_DENSITY, ST_CORECORE, ST_PURIFY, ST_SWEEPS, ST_BIPARTITE, ST_FULLJAC,
             ST_PURIFY_PRODUCTS, kStageSlots };
constexpr int kTimedSlots = ST_PURIFY + 1;  // slots [0, kTimedSlots) are cycles, the rest counts

struct StageClock {
  unsigned long long* out;
  long long t;
  __device__ __forceinline__ void start() { if (out) t = clock64(); }
  __device__ __forceinline__ void lap(int slot) {
    if (out) {
      const long long now = clock64();
      if (threadIdx.x == 0) out[slot] += (unsigned long long)(now - t);
      t = now;
    }
  }
  __device__ __forceinline__ void add(int slot, unsigned long long v) {
    if (out && threadIdx.x == 0) out[slot] += v;
  }
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

enum : int { STAGE_INTS = 1, STAGE_HCORE = 2, STAGE_SCF = 4, STAGE_CC = 8, STAGE_ALL = 15,
             STAGE_FOCK = 16 /* F and E_el from the P already in device memory */ };

enum : int { MOL_OK = 0, MOL_EIG_FAILED = 1, MOL_NAN = 2 };

// SOLVER_PURIFY_MIXED: as SOLVER_PURIFY, with the products in FP32 until the recursion is near
// idempotent, FP64 after: on the tensor cores (tcgen05 kind::tf32, split in two TF32 parts) for
// one-CTA molecules of nao 65-128, as FP32 SSYRK on the grid path; other sizes keep FP64.
enum : int { SOLVER_PURIFY = 0, SOLVER_JACOBI = 1, SOLVER_PURIFY_MIXED = 2 };

__host__ __device__ inline int smem_ld(int n) { return n | 1; }

// Shared memory plan.  The matrix region holds G (n x ld, column-major) and, when it fits, the
// eigenvectors V (n x ld) too; otherwise V stays in global memory.  The region size is fixed
// per launch (mat_doubles); the small arrays follow it.
constexpr int kVsmemMax = 110;  // 2 * 110 * 111 doubles = 195 KB: G and V both in smem

// Jacobi thresholds, absolute in eV (Fock elements are O(1..100) eV): rotations below
// kJacobiRotAbs are skipped; sweeps end after one whose largest off-diagonal was below
// kJacobiDoneAbs, which leaves occupied-virtual couplings of order 1e-14 / gap.
constexpr double kJacobiRotAbs = 1e-12;
constexpr double kJacobiDoneAbs = 1e-7;

// The first eigensolve of an SCF (no previous vectors) rotates every pair.  Later ones rotate
// occupied-virtual pairs only and are accepted when the largest
// occupied Rayleigh quotient stays kCrossMargin eV below the smallest virtual one (the
// quotients differ from eigenvalues by the small within-block couplings left unrotated);
// otherwise a full Jacobi follows, so the occupied set is always the nocc lowest states.
constexpr int kFullJacobiSteps = 1;
constexpr double kCrossMargin = 1.0;
// Occupied-virtual couplings sit across a gap of at least kCrossMargin, where Jacobi converges
// quadratically: after a sweep whose largest coupling was below kJacobiDoneGapped the next
// would start below n * 3e-6^2 / 1 eV ~ 1e-9 eV (n <= 160), so no confirmation sweep is run.
constexpr double kJacobiDoneGapped = 3e-6;

// Largest nao whose work matrix fits one CTA's shared memory; above it the work matrices (and
// V) are in global memory.
constexpr int kGsmemMax = 160;

// The Fock build keeps its staging buffers and heavy-heavy partial sums in the matrix region
// while G (and X) are dead: from its start, or after G and V when G's part is too small (V,
// in shared memory up to nao 110, must survive).  Above nao 160 the partial sums go to the
// global work matrix instead.
__host__ __device__ inline size_t fock_smem_doubles(int n) {
  return (size_t)kFockStage + (n > kGsmemMax ? 0 : fock_xx_doubles(n));
}
__host__ __device__ inline size_t fock_stage_at(int n) {
  const size_t g = (size_t)n * smem_ld(n);
  return (n > kGsmemMax || n > kVsmemMax || g >= fock_smem_doubles(n)) ? 0 : 2 * g;
}

__host__ __device__ inline size_t mat_doubles_for(int n) {
  const size_t ld = (size_t)smem_ld(n);
  if (n > kGsmemMax) return kFockStage;
  const size_t jac = (n <= kVsmemMax ? 2 : 1) * (size_t)n * ld;
  const size_t pur = purify_doubles(n);  // the purification's X shares the region
  const size_t fk = fock_stage_at(n) + fock_smem_doubles(n);
  const size_t m = jac > pur ? jac : pur;
  return m > fk ? m : fk;
}

__host__ __device__ inline size_t extra_doubles(int nmax) {
  return 2 * (3 * (size_t)nmax + 8)  // wq and J (each <= 2.5 n) + pad
         + (size_t)nmax          // eigenvalues of the last eigensolve
         + 64                    // reductions (two halves of 32)
         + (size_t)nmax + 2      // occupied and virtual index lists (ints, two per double)
         + (size_t)nmax / 8 + 2; // heavy atom list of the Fock build (ints)
}

__device__ __forceinline__ MolView make_view(const BatchArgs& a, const MolDesc& d) {
  MolView v;
  v.natoms = d.natoms; v.nao = d.nao; v.nocc = d.nocc;
  v.slot = a.slot + d.atom0;
  v.pos = a.pos + 3 * d.atom0;
  v.first = a.first + d.atom0;
  v.row_off = a.row_off + d.atom0;
  v.hb = a.hb + d.atom0;
  v.ints = a.ints + d.blk0;
  v.H = a.H + d.pk0; v.P = a.P + d.pk0; v.F = a.F + d.pk0;
  v.V = a.V + d.sq0; v.T = a.T + d.sq0;
  v.eig = a.eig + d.ao0;
  v.W = a.W ? a.W + d.w0 : nullptr;
  return v;
}

// P (packed) = 2 Vo Vo^T with Vo = nocc column vectors (column-major, ldo) in shared memory;
// 4x4 register tiles over the lower triangle of tiles.
// With damping d > 0 the new density is mixed with the previous one still in P:
// P = (1 - d) 2 Vo Vo^T + d P.
__device__ inline void block_density(int n, int nocc, const double* Vo, int ldo, double* P,
                                     double d) {
  const int tiles = (n + 3) >> 2;
  const int ntile = tiles * (tiles + 1) / 2;
  for (int t = threadIdx.x; t < ntile; t += blockDim.x) {
    int ti, tj;
    {
      int a = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
      while ((a + 1) * (a + 2) / 2 <= t) ++a;
      while (a * (a + 1) / 2 > t) --a;
      ti = a; tj = t - a * (a + 1) / 2;
    }
    const int i0 = ti * 4, j0 = tj * 4;
    double acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
    for (int k = 0; k < nocc; ++k) {
      const double* col = Vo + (int64_t)k * ldo;
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

// rank of dval[i] in ascending order (ties by index)
__device__ __forceinline__ int ascending_rank(const double* dval, int n, int i) {
  const double di = dval[i];
  int rank = 0;
  for (int j = 0; j < n; ++j) {
    const double dj = dval[j];
    rank += (dj < di) || (dj == di && j < i);
  }
  return rank;
}

// occ <- indices of the nocc smallest dval (in ascending order), vir <- the rest (ascending)
__device__ inline void split_by_rank(const double* dval, int n, int nocc, int* occ, int* vir) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int rank = ascending_rank(dval, n, i);
    if (rank < nocc) occ[rank] = i;
    else vir[rank - nocc] = i;
  }
}

// PLACE: 0 = G and V in shared memory (nao <= kVsmemMax), 1 = G in shared memory and V in
// global memory (nao <= kGsmemMax), 2 = both in global memory (larger; CR must be 0).  A
// template parameter so every access in the eigensolver has a known address space.
// ---- Pulay DIIS on the batched path (kernel instances with FEAT_DIIS; off by default) ----
// The last diis_depth Fock matrices F_out(P_k) and their residuals e_k = F_out(P_k) - F_in,k
// (F_in,k the matrix P_k was purified from) are kept in global memory; B_ij = <e_i, e_j>.  After
// each Fock build the next density is purified from F = sum c_i F_out,i with
// [B 1; 1 0] (c, -lambda) = (0, 1), solved by one thread (Gaussian elimination with partial
// pivoting, B scaled by its largest diagonal); a singular system or a coefficient beyond 1e6
// keeps the plain F.  The solve is the grid path's (capi.cu diis_step); the error vector is the
// Fock residual (Pulay mixing of Fock matrices) instead of the commutator F P - P F, which
// would need a dense product per step: with it each step cost 1.7x, more than the 38 % fewer
// steps saved.  Both vanish at self-consistency.
constexpr int kDiisMaxDepth = 8;
constexpr int kDiisB = kDiisMaxDepth * kDiisMaxDepth;

// Where a molecule's DIIS history starts: depth F_out, depth residuals, then F_in.
__device__ __forceinline__ double* diis_history(const BatchArgs& a, int64_t sq0) {
  return a.diis + (2 * (int64_t)a.diis_depth + 1) * sq0;
}

template <int NT>
__device__ __noinline__ void block_diis(const BatchArgs& a, int64_t sq0, const MolView& m,
                                        int mi, double* Ffull, int& count, int& next,
                                        double* red) {
  const int n = m.nao, depth = a.diis_depth;
  const int64_t nn = (int64_t)n * n;
  double* Fh = diis_history(a, sq0);
  double* Eh = Fh + (int64_t)depth * nn;
  double* Fin = Eh + (int64_t)depth * nn;
  double* B = a.diis_B + (int64_t)mi * kDiisB;
  const int slot = next;
  double* Fs = Fh + slot * nn;
  double* Es = Eh + slot * nn;
  for (int64_t t = threadIdx.x; t < nn; t += NT) {
    const double f = Ffull[t];
    Fs[t] = f;
    Es[t] = f - Fin[t];
  }
  __syncthreads();
  count = count + 1 < depth ? count + 1 : depth;
  next = (slot + 1) % depth;
  for (int jj = 0; jj < count; ++jj) {
    const double* Ej = Eh + jj * nn;
    double s = 0.0, unused = 0.0;
    for (int64_t t = threadIdx.x; t < nn; t += NT) s = fma(Es[t], Ej[t], s);
    block_sum2<NT>(s, unused, red);
    if (threadIdx.x == 0) B[slot * kDiisMaxDepth + jj] = B[jj * kDiisMaxDepth + slot] = s;
  }
  __syncthreads();
  const int mm = count;
  if (mm < 2) {
    for (int64_t t = threadIdx.x; t < nn; t += NT) Fin[t] = Ffull[t];
    __syncthreads();
    return;
  }
  if (threadIdx.x == 0) {
    double A[kDiisMaxDepth + 1][kDiisMaxDepth + 2];
    double scale = 0.0;
    for (int i = 0; i < mm; ++i) scale = fmax(scale, B[i * kDiisMaxDepth + i]);
    bool ok = scale > 0.0;
    for (int i = 0; i <= mm; ++i)
      for (int k = 0; k <= mm + 1; ++k) A[i][k] = 0.0;
    for (int i = 0; i < mm && ok; ++i) {
      for (int j = 0; j < mm; ++j) A[i][j] = B[i * kDiisMaxDepth + j] / scale;
      A[i][mm] = A[mm][i] = 1.0;
    }
    A[mm][mm + 1] = 1.0;
    for (int c = 0; c <= mm && ok; ++c) {
      int piv = c;
      for (int r = c + 1; r <= mm; ++r)
        if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
      if (!(fabs(A[piv][c]) > 1e-14)) { ok = false; break; }
      for (int k = 0; k <= mm + 1; ++k) {
        const double t = A[c][k];
        A[c][k] = A[piv][k];
        A[piv][k] = t;
      }
      for (int r = 0; r <= mm; ++r) {
        if (r == c) continue;
        const double f = A[r][c] / A[c][c];
        for (int k = c; k <= mm + 1; ++k) A[r][k] -= f * A[c][k];
      }
    }
    for (int i = 0; i < mm && ok; ++i) {
      red[i] = A[i][mm + 1] / A[i][i];
      if (!(fabs(red[i]) < 1e6)) ok = false;
    }
    red[kDiisMaxDepth] = ok ? 1.0 : 0.0;
  }
  __syncthreads();
  const bool ok = red[kDiisMaxDepth] != 0.0;
  double c[kDiisMaxDepth];
#pragma unroll
  for (int i = 0; i < kDiisMaxDepth; ++i) c[i] = i < mm ? red[i] : 0.0;
  __syncthreads();  // red is reused by the next reduction
  for (int64_t t = threadIdx.x; t < nn; t += NT) {
    double f = Ffull[t];
    if (ok) {
      f = 0.0;
      for (int i = 0; i < mm; ++i) f = fma(c[i], Fh[i * nn + t], f);
      Ffull[t] = f;
    }
    Fin[t] = f;  // the matrix the next density is purified from
  }
  __syncthreads();
}

// Kernel feature bits (template FEAT): the tensor-core mixed form may be taken, DIIS is on.
// Instances without a bit carry no call into its code (a call changes the register
// allocation of the whole kernel).
enum : int { FEAT_TENSOR = 1, FEAT_DIIS = 2 };

template <int NT, int CR, int PLACE, int MX>
__device__ void run_molecule(const BatchArgs& a, int mi, double* smem) {
  const MolDesc d = a.mols[mi];
  const MolView m = make_view(a, d);
  const int n = m.nao, ld = PLACE == 2 ? n : smem_ld(n);
  const size_t nmax = (size_t)a.nmax;
  double* G = PLACE == 2 ? m.W : smem;
  double* V = PLACE == 0 ? smem + (size_t)n * ld : m.V;
  const int ldv = PLACE == 0 ? ld : n;
  double* wq = smem + a.mat_doubles;
  double* Jc = wq + 3 * nmax + 8;  // Coulomb sums of the Fock build
  double* dval = Jc + 3 * nmax + 8;
  double* stage = smem + fock_stage_at(n);
  double* xs = PLACE == 2 ? m.W : stage + kFockStage;
  double* red = dval + nmax;
  int* occ = reinterpret_cast<int*>(red + 64);
  int* vir = occ + nmax + 2;
  int* hv = vir + nmax + 2;
  double* Ffull = m.T;  // F as a full n x n matrix, global scratch
  if (a.t_begin && threadIdx.x == 0) a.t_begin[mi] = global_ns();
  StageClock clk{a.stage_cycles ? a.stage_cycles + (int64_t)mi * kStageSlots : nullptr, 0};
  if (clk.out && threadIdx.x == 0)
    for (int k = 0; k < kStageSlots; ++k) clk.out[k] = 0;
  clk.start();

  if (a.stages & STAGE_INTS) {
    block_integrals(m);
    __syncthreads();
    clk.lap(ST_INTS);
  }
  if (a.stages & STAGE_HCORE) {
    block_hcore(m);
    __syncthreads();
    clk.lap(ST_HCORE);
  }
  double E = 0.0;
  int steps = 0, conv = 0, status = MOL_OK;
  if (a.stages & STAGE_SCF) {
    block_guess(m);
    __syncthreads();
    E = block_fock_energy<NT>(m, Ffull, n, wq, Jc, stage, xs, hv, red);
    clk.lap(ST_FOCK);
    if (a.hist && threadIdx.x == 0) a.hist[(int64_t)mi * a.hist_stride] = E;
    if (E != E) status = MOL_NAN;  // non-finite input (e.g. a NaN coordinate): no SCF step
    // purification needs X in shared memory (nao <= 160); larger molecules diagonalise
    const bool purify = a.solver != SOLVER_JACOBI;
    int diis_count = 0, diis_next = 0;
    if constexpr ((MX & FEAT_DIIS) != 0) {
      if (a.diis_depth >= 2) {  // F_in of the first step: the guess Fock matrix
        double* Fin = diis_history(a, d.sq0) + 2 * (int64_t)a.diis_depth * n * n;
        for (int t = threadIdx.x; t < n * n; t += blockDim.x) Fin[t] = Ffull[t];
        __syncthreads();
      }
    }
    while (status == MOL_OK && !conv && steps < a.max_iter) {
      bool cold = steps == 0, jacobi = !purify;
      if (purify) {
        // ---- P from F by purification; a Jacobi eigensolve if that fails ----
        int prod = -1;
        const double* Xr = smem;
        if constexpr (PLACE == 2) {  // X and its partner in the global work matrix
          double* Xo = nullptr;
          if constexpr (NT == BpCfg::THREADS) {
            if (a.wmaps && d.wmap >= 0) {
              // TMA-staged tiles; the ring follows the kernel's other shared memory
              unsigned char* ring = reinterpret_cast<unsigned char*>(
                  smem + a.mat_doubles + extra_doubles(a.nmax));
              const CUtensorMap* maps = a.wmaps + kWorkMaps * d.wmap;
              bool tensor = false;
              if constexpr ((MX & FEAT_TENSOR) != 0) {
                // mixed form: TF32 tensor-core phase, FP64 finish
                tensor = a.solver == SOLVER_PURIFY_MIXED;
                if (tensor)
                  prod = block_purify_tiles32<NT>(Ffull, n, m.nocc, m.W, m.W + purify_doubles(n),
                                                  maps, ring, wq, red, &Xo, a.wait_spins);
              }
              if (!tensor)
                prod = block_purify_tiles<NT>(Ffull, n, m.nocc, m.W, m.W + purify_doubles(n),
                                              maps, maps + 1, ring, wq, red, &Xo, a.wait_spins);
            } else {
              prod = block_purify_global<NT>(Ffull, n, m.nocc, m.W, m.W + purify_doubles(n), wq,
                                             red, &Xo);
            }
          } else {
            prod = block_purify_global<NT>(Ffull, n, m.nocc, m.W, m.W + purify_doubles(n), wq, red,
                                           &Xo);
          }
          Xr = Xo;
        } else {
          bool tensor = false;
          if constexpr ((MX & FEAT_TENSOR) && NT == 512) {
            // mixed form: TF32 tensor-core products (tcgen05), FP64 finish; X's region holds
            // the split copies (2 x max(128, n16) x n16 floats)
            const int n16 = purify_n16(n);
            tensor = a.solver == SOLVER_PURIFY_MIXED && n16 > 64 && n16 <= 160 &&
                     (size_t)(n16 > 128 ? n16 : 128) * n16 <= a.mat_doubles;
            if (tensor)
              prod = block_purify_mixed<NT>(Ffull, n, m.nocc, smem, wq, red, a.wait_spins);
          }
          if (!tensor) prod = block_purify<NT>(Ffull, n, m.nocc, smem, wq, red);
        }
        clk.lap(ST_PURIFY);
        clk.add(ST_PURIFY_PRODUCTS, (unsigned long long)(prod > 0 ? prod : 0));
        if (prod >= 0) {
          purify_density(Xr, n, m.P, a.damping);
          __syncthreads();
          clk.lap(ST_DENSITY);
        } else {
          jacobi = cold = true;
        }
      }
      if (jacobi) {
        // ---- eigensolve of F: Jacobi on V^T F V through (V, G = F V), V warm-started ----
        if (cold) {
          for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
            const int j = t / n, i = t % n;
            V[(int64_t)j * ldv + i] = i == j ? 1.0 : 0.0;
            G[(int64_t)j * ld + i] = Ffull[t];
          }
        } else {
          block_shifted_product(n, Ffull, 0.0, V, ldv, G, ld);
        }
        __syncthreads();
        clk.lap(ST_SHIFT_GEMM);
        const int nocc = m.nocc, nvir = n - nocc;
        int sw;
        bool full = cold || steps < kFullJacobiSteps || a.sorted_vectors || nocc == 0 || nvir == 0;
        if (!full) {
          // occupied / virtual split of the warm-started columns by their Rayleigh quotients
          block_rayleigh<NT>(n, G, ld, V, ldv, 0.0, dval);
          __syncthreads();
          split_by_rank(dval, n, nocc, occ, vir);
          __syncthreads();
          const bool o_small = nocc <= nvir;
          sw = block_jacobi_fv<NT, CR>(n, G, ld, V, ldv, red, kJacobiRotAbs, kJacobiDoneGapped,
                                       a.max_sweeps,
                                       o_small ? occ : vir, o_small ? nocc : nvir,
                                       o_small ? vir : occ, o_small ? nvir : nocc);
          if (sw >= 0) {
            clk.add(ST_BIPARTITE, 1);
            // the occupied block must still hold the lowest states (no level crossing)
            block_rayleigh<NT>(n, G, ld, V, ldv, 0.0, dval);
            __syncthreads();
            double hi = -INFINITY, lo = INFINITY;
            for (int i = threadIdx.x; i < nocc; i += blockDim.x) hi = fmax(hi, dval[occ[i]]);
            for (int i = threadIdx.x; i < nvir; i += blockDim.x) lo = fmin(lo, dval[vir[i]]);
            hi = block_max<NT>(hi, red);
            lo = -block_max<NT>(-lo, red);
            full = !(hi + kCrossMargin < lo);
          }
        }
        if (full) {
          clk.add(ST_FULLJAC, 1);
          sw = block_jacobi_fv<NT, CR>(n, G, ld, V, ldv, red, kJacobiRotAbs, kJacobiDoneAbs,
                                       a.max_sweeps);
          if (sw >= 0) {
            block_rayleigh<NT>(n, G, ld, V, ldv, 0.0, dval);
            __syncthreads();
            split_by_rank(dval, n, nocc, occ, vir);
          }
        }
        clk.lap(ST_JACOBI);
        clk.add(ST_SWEEPS, (unsigned long long)(sw > 0 ? sw : 0));
        if (sw < 0) { status = MOL_EIG_FAILED; break; }
        __syncthreads();
        clk.lap(ST_EIGVAL_SORT);
        // ---- density from the occupied vectors, gathered into the G region ----
        for (int t = threadIdx.x; t < n * m.nocc; t += blockDim.x) {
          const int k = t / n, i = t % n;
          G[(int64_t)k * ld + i] = V[(int64_t)occ[k] * ldv + i];
        }
        __syncthreads();
        block_density(n, m.nocc, G, ld, m.P, a.damping);
        __syncthreads();
        clk.lap(ST_DENSITY);
      }
      // the F just diagonalised, kept for the eigenpairs reported at the end
      if (purify && a.sorted_vectors) {
        for (int t = threadIdx.x; t < n * n; t += blockDim.x) m.V[t] = Ffull[t];
        __syncthreads();
      }
      // ---- Fock + energy ----
      const double Eold = E;
      E = block_fock_energy<NT>(m, Ffull, n, wq, Jc, stage, xs, hv, red);
      clk.lap(ST_FOCK);
      ++steps;
      if (a.hist && threadIdx.x == 0) a.hist[(int64_t)mi * a.hist_stride + steps] = E;
      if (E != E) { status = MOL_NAN; break; }
      conv = fabs(Eold - E) < a.tol;
      if constexpr ((MX & FEAT_DIIS) != 0) {
        if (!conv && steps < a.max_iter && a.diis_depth >= 2 && status == MOL_OK)
          block_diis<NT>(a, d.sq0, m, mi, Ffull, diis_count, diis_next, red);
      }
    }
    if (purify && a.sorted_vectors && steps > 0 && status == MOL_OK) {
      // eigenpairs of the last F that produced a density (saved in m.V): one full Jacobi
      for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
        const int j = t / n, i = t % n;
        G[(int64_t)j * ld + i] = m.V[t];
      }
      __syncthreads();
      for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
        const int j = t / n, i = t % n;
        V[(int64_t)j * ldv + i] = i == j ? 1.0 : 0.0;
      }
      __syncthreads();
      clk.start();
      clk.add(ST_FULLJAC, 1);
      const int sw = block_jacobi_fv<NT, CR>(n, G, ld, V, ldv, red, kJacobiRotAbs, kJacobiDoneAbs,
                                             a.max_sweeps);
      clk.add(ST_SWEEPS, (unsigned long long)(sw > 0 ? sw : 0));
      if (sw < 0) status = MOL_EIG_FAILED;
      else block_rayleigh<NT>(n, G, ld, V, ldv, 0.0, dval);
      __syncthreads();
      clk.lap(ST_JACOBI);
    }
    // eigenvalues (ascending) and, on request, the eigenvectors sorted the same way into T
    // (column k = vector k, the layout of SCFCalculation::eigenVec); with purification only
    // when requested (dval is not computed otherwise)
    if (steps > 0 && (!purify || a.sorted_vectors) && status == MOL_OK) {
      __syncthreads();
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int rank = ascending_rank(dval, n, i);
        m.eig[rank] = dval[i];
        if (a.sorted_vectors)
          for (int r = 0; r < n; ++r) m.T[(int64_t)rank * n + r] = V[(int64_t)i * ldv + r];
      }
    }
  }
  if (a.stages & STAGE_FOCK) {
    E = block_fock_energy<NT>(m, nullptr, 0, wq, Jc, stage, xs, hv, red);
    if (threadIdx.x == 0) a.e_el[mi] = E;
  }
  double ecc = 0.0;
  if (a.stages & STAGE_CC) {
    clk.start();
    ecc = block_core_core<NT>(m, red);
    clk.lap(ST_CORECORE);
  }
  if (threadIdx.x == 0) {
    if (a.stages & STAGE_SCF) {
      a.e_el[mi] = E;
      a.n_iter[mi] = steps;
      a.converged[mi] = conv;
      a.status[mi] = status;
    }
    if (a.stages & STAGE_CC) a.e_cc[mi] = ecc;
    if (a.t_end) a.t_end[mi] = global_ns();
  }
  __syncthreads();
}

// NT threads per CTA; CR column registers per lane in the eigensolver (nao <= 32 * CR).
// MX: FEAT_* bits -- FEAT_TENSOR: the instance that can take the tensor-core mixed form
// (launched only for that solver); FEAT_DIIS: the instance with DIIS (launched only with it
// on).  The default instances (MX = 0) carry no call into either.
template <int NT, int CR, int MX = 0>
__global__ void __launch_bounds__(NT, 512 / NT) k_batch_scf(BatchArgs a) {
  extern __shared__ double smem[];
  __shared__ int s_next;
  for (;;) {
    if (threadIdx.x == 0) s_next = atomicAdd(a.counter, 1);
    __syncthreads();
    const int q = s_next;
    __syncthreads();
    if (q >= a.nmol) break;
    const int mi = a.order[q];
    const int n = a.mols[mi].nao;
    if constexpr (CR == 0) {
      run_molecule<NT, 0, 2, MX>(a, mi, smem);
    } else {
      if (n <= kVsmemMax)
        run_molecule<NT, CR, 0, MX>(a, mi, smem);
      else
        run_molecule<NT, CR, 1, MX>(a, mi, smem);
    }
  }
}

}  // namespace sgb
