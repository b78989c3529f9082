/* semigpu_b200 — C ABI of the B200 MNDO SCF engine.
 *
 * Plain pointers and sizes only.  Every call returns an int status: 0 on success, < 0 on an
 * error (see SGB_E_*), and sgb_last_error() gives the message.  A context owns one CUDA stream
 * on one device; molecule and batch handles own their device memory; all host buffers are the
 * caller's.  Calls on one context are not thread-safe (one host thread per context, as the
 * reference's single-threaded driver).
 *
 * Units follow the reference: coordinates in Angstrom on input (converted to bohr with
 * 1.8897259886, mymath.h:84-87), energies and matrix elements in eV.  Matrices are packed
 * lower triangles, element (i,j) with i >= j at i*(i+1)/2 + j (mymemory.cpp:369-371); the AO
 * order is atoms in input order, one s AO for H and s, px, py, pz for C, N, O
 * (atomicOrbitals.cpp:76-119).  Reference paths are under src/common/ of
 * LuisAlfredoNu/semiGPU.
 */
#ifndef SEMIGPU_B200_H
#define SEMIGPU_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------- */
#define SGB_OK 0
#define SGB_E_ARG -1          /* invalid argument (null pointer, bad size, bad enum)        */
#define SGB_E_ELEMENT -2      /* element without MNDO parameters (only H, C, N, O)           */
#define SGB_E_CUDA -3         /* CUDA runtime error (message in sgb_last_error)              */
#define SGB_E_NOMEM -4        /* device allocation failed or over the context's HBM budget  */
#define SGB_E_STATE -5        /* stage called out of order (e.g. Hcore before integrals)     */
#define SGB_E_UNSUPPORTED -6  /* size outside what this build handles                        */
#define SGB_E_EIG 1           /* SCF stopped: eigensolver did not converge (as LAPACK info>0)*/
#define SGB_E_NAN 2           /* SCF stopped: non-finite energy                              */
#define SGB_E_NOCONV 3        /* sgb_gradient: a geometry's SCF reached max_iter unconverged */

/* ---- matrices that can be read back ----------------------------------------------------- */
#define SGB_BLOCKS 0  /* integral blocks, the reference's ragged [A][B<=A] array flattened   */
#define SGB_HCORE 1   /* packed Hcore                                                        */
#define SGB_FOCK 2    /* packed Fock matrix of the last SCF step                             */
#define SGB_DENSITY 3 /* packed density matrix of the last SCF step                          */
#define SGB_EIGVAL 4  /* nao eigenvalues of the last eigensolve, ascending                   */
#define SGB_EIGVEC 5  /* nao x nao eigenvectors, column-major (column k = vector k), the    */
                      /* layout of SCFCalculation::eigenVec                                  */

typedef struct sgb_ctx sgb_ctx;
typedef struct sgb_mol sgb_mol;
typedef struct sgb_batch sgb_batch;

typedef struct {
  double e_el;    /* electronic energy (SCFCalculation::finalEnergy)                     */
  int n_iter;     /* SCF steps taken                                                      */
  int converged;  /* |dE| < tol reached (SCFCalculation::energyConverge)                  */
  int status;     /* SGB_OK, SGB_E_EIG or SGB_E_NAN                                        */
} sgb_scf_result;

/* ---- context ---------------------------------------------------------------------------- */
/* Binds a device, loads the MNDO tables, creates the stream.  hbm_budget_bytes = 0: no limit
 * beyond the device's own. */
int sgb_ctx_create(int device, size_t hbm_budget_bytes, sgb_ctx **out);
/* Frees the context's device and pinned host memory, streams and events.  Molecules and
 * batches still alive lose their device memory here and stay valid only for their own destroy
 * call (which then frees their host part alone). */
int sgb_ctx_destroy(sgb_ctx *ctx);
int sgb_ctx_synchronize(sgb_ctx *ctx);
const char *sgb_last_error(const sgb_ctx *ctx);
const char *sgb_status_string(int status);
/* How an SCF step gets the density P from F (no counterpart in the reference, which always
 *   diagonalises with LAPACK dsyev, scfcalculation.cpp:94-110):
 *   SGB_SOLVER_PURIFY (default) -- trace-correcting purification on the FP64 tensor cores (the
 *     same aufbau projector; a Jacobi eigensolve replaces it for a step where it does not
 *     converge, and gives the eigenpairs when they are asked for);
 *   SGB_SOLVER_JACOBI -- warm-started Jacobi eigensolves every step;
 *   SGB_SOLVER_PURIFY_MIXED -- the mixed-precision form: the purification products run on the
 *     tcgen05 tensor cores at FP32-level accuracy (TF32, X split in two parts) until the
 *     recursion is near idempotent and finish in FP64 (Fock, energies and the convergence test
 *     stay FP64), for batched molecules above 64 AOs (below, FP64 products throughout) and for
 *     one molecule on the whole GPU from about 2000 AOs (below, FP64 products with the mixed
 *     form's earlier exit); results within 1e-4 eV of the FP64 form.
 * The environment variable SGB_DENSITY_SOLVER=jacobi or =mixed changes the default (also for
 * sgb_scf_noalloc). */
#define SGB_SOLVER_PURIFY 0
#define SGB_SOLVER_JACOBI 1
#define SGB_SOLVER_PURIFY_MIXED 2
int sgb_ctx_set_density_solver(sgb_ctx *ctx, int solver);
/* The size classes of the batched launch (no counterpart in the reference): *count classes,
 * class k takes molecules up to nao_max[k] AOs and launches CTAs of threads[k] threads by
 * default (arrays of max_count entries; either may be NULL).  sgb_ctx_set_class_threads sets
 * the CTA size per class for this context (128 only for the classes up to nao 64, 512 for the
 * large-molecule class); semigpu_b200/autotune.py picks them by timing. */
int sgb_size_classes(int *count, int *nao_max, int *threads, int max_count);
int sgb_ctx_set_class_threads(sgb_ctx *ctx, int count, const int *threads);
/* Tile configurations of the whole-GPU FP64 purification (one large molecule, sgb_scf above
 * nao 160; no counterpart in the reference): *count configurations, configuration k has
 * bm[k] x bm[k] tiles, warps[k] warps per CTA, kblocks[k] k-blocks of 16 doubles per TMA ring
 * stage and stages[k] stages (arrays of max_count entries; any may be NULL).
 * sgb_ctx_set_grid_config fixes the configuration for this context's single-molecule SCF runs
 * (-1, the default: chosen by size -- the largest tile that gives every SM work);
 * semigpu_b200/autotune.py tune_grid picks one by timing an SCF step. */
int sgb_grid_configs(int *count, int *bm, int *warps, int *kblocks, int *stages, int max_count);
int sgb_ctx_set_grid_config(sgb_ctx *ctx, int config);
/* Caps the batched launches of this context at share x (number of SMs) CTAs' worth of SMs
 * (0 < share <= 1; 1 = the whole GPU, the default).  No counterpart in the reference; a
 * server running several contexts side by side uses it so that one context's persistent
 * launch of long (large-molecule) work leaves SMs to the others. */
int sgb_ctx_set_sm_share(sgb_ctx *ctx, double share);
/* Pulay DIIS of depth 2..8 (0 = off, the default) for every SCF of this context: F is
 * extrapolated from the last `depth` Fock matrices: on the grid path by the host, with the
 * commutator FP - PF as error; in the batched launches, and single molecules on one CTA, by
 * each molecule's CTA, with the Fock residual F(P_k) - F_k as error (no dense product per step)
 * and (2 depth + 1) nao^2 doubles of history per molecule allocated on the first such launch.
 * It changes the SCF trajectory, so step counts no longer follow the reference's, and the
 * converged energy agrees with the plain loop's only to the SCF tolerance (on the 4096-molecule
 * bench batch at 1e-6 eV: up to 1.2e-6 eV apart, both loops having stopped at |dE| < 1e-6), not
 * to the 1e-6 eV parity of the default loop.  Next step after the reference's SCF loop
 * (scfcalculation.cpp:82-141), which has no convergence acceleration. */
int sgb_ctx_set_diis(sgb_ctx *ctx, int depth);
/* Density damping 0 <= factor < 1 (0 = off, the default) for every SCF of this context: the
 * density that enters each Fock build is P = (1 - factor) P_new + factor P_previous.  Next step
 * after the reference's SCF loop (scfcalculation.cpp:82-141), which takes P_new as is; it
 * changes the SCF trajectory (damped oscillations), and the converged energy is the same. */
int sgb_ctx_set_damping(sgb_ctx *ctx, double factor);
/* Limits of the engine's bounded loops for this context (no counterpart in the reference,
 * whose only bound is LAPACK's own, scfcalculation.cpp:87-93).  max_sweeps: Jacobi sweeps per
 * eigensolve (0 = the default: 40 on one CTA, 60 on the grid path); an eigensolve that does not
 * converge within it stops that molecule's SCF with SGB_E_EIG.  wait_spins: polls of each
 * bounded device wait -- the first wait for a product's tensor-core MMAs (a timed-out wait
 * abandons the purification of that SCF step, which is then diagonalised) and the grid-path
 * barriers (a timed-out barrier ends the launch with SGB_E_CUDA); < 0 = the default bounds
 * (hundreds of milliseconds to seconds).  Small values are for tests of those failure paths. */
int sgb_ctx_set_limits(sgb_ctx *ctx, int max_sweeps, long long wait_spins);
/* Failure-path check of the bounded grid barrier (no counterpart in the reference): launches
 * `blocks` co-resident blocks (at most one per SM) at one barrier that expects blocks + extra
 * arrivals; with extra > 0 it can never complete, so every block gives up after `spins` polls
 * (>= 64 ns each) and the kernel ends.  *timed_out = 1 when the barrier reported its timeout. */
int sgb_diag_barrier_timeout(sgb_ctx *ctx, int blocks, int extra, long long spins,
                             int *timed_out);
/* Reserves a reusable device arena of `bytes` for this context: a batch that fits is built in
 * it instead of allocating, and releasing the batch does not free device memory (cudaFree
 * synchronises the whole device, which would stall other contexts' work).  One batch at a time
 * uses the arena; bytes = 0 releases it. */
int sgb_ctx_reserve(sgb_ctx *ctx, size_t bytes);
/* Launch priority of the context's work: high != 0 puts its streams at the device's greatest
 * stream priority, 0 at the default.  When the SMs are busy with another context's long
 * persistent launches, the hardware then hands this context's blocks to the next free SMs
 * before the other launches' waiting blocks (a serving loop gives its small-molecule workers
 * high priority).  Waits for the context's queued work, then replaces its streams. */
int sgb_ctx_set_priority(sgb_ctx *ctx, int high);
/* Bytes of device memory currently held by the context: its molecules and batches, and the
 * arenas of destroyed ones that it keeps for reuse (at most 16 of them and 8 GiB; released
 * when the budget or a failed allocation needs the room, and by sgb_ctx_destroy). */
size_t sgb_ctx_bytes_in_use(const sgb_ctx *ctx);

/* ---- MNDO element data ------------------------------------------------------------------ */
/* Parameters of element Z (1, 6, 7, 8) as used by the engine, in the units of
 * MNDO_parameters.cpp:47-122 (eV, bohr, 1/Angstrom, kcal/mol).  Replaces reading the public
 * arrays of MNDOparameter. */
#define SGB_P_USS 0
#define SGB_P_UPP 1
#define SGB_P_ZS 2
#define SGB_P_BETAS 3
#define SGB_P_BETAP 4
#define SGB_P_ALPHA 5
#define SGB_P_GSS 6
#define SGB_P_GPP 7
#define SGB_P_GSP 8
#define SGB_P_GP2 9
#define SGB_P_HSP 10
#define SGB_P_DD1 11
#define SGB_P_DD2 12
#define SGB_P_RHO0 13
#define SGB_P_RHO1 14
#define SGB_P_RHO2 15
#define SGB_P_HEAT 16
#define SGB_P_EISOL 17
#define SGB_PARAM_COUNT 18
int sgb_mndo_parameters(int Z, double *values);
/* Heat of formation (kcal/mol) from a total energy (eV, electronic + core-core), MOPAC's
 * convention: (E_tot - sum_A E_isol(A)) * 23.060548 + sum_A dH_f(atom A), with the atomic
 * E_isol ("eisol") and dH_f ("heat") of MNDO_parameters.cpp:47-122, which the reference stores
 * but never uses.  Host arithmetic only; no counterpart in the reference's SCF path. */
int sgb_heat_of_formation(int natoms, const int *Z, double e_tot, double *dhf_kcal);

/* ---- one molecule: the reference's stage API ------------------------------------------- */
/* Replaces ReadXYZFile output handling + ListAtomicOrbitals::SetOrbitals
 * (atomicOrbitals.cpp:76-119) + TwoCenterIntegral::Alloc4AllTwoCenterIntegral
 * (twocenterintegral.cpp:55-107): validates the elements, builds the AO table and allocates
 * integral blocks, Hcore, SCF matrices on the device.  Z: natoms atomic numbers; xyz:
 * natoms*3 Cartesian coordinates in Angstrom. */
int sgb_mol_create(sgb_ctx *ctx, int natoms, const int *Z, const double *xyz, sgb_mol **out);
int sgb_mol_destroy(sgb_mol *mol);
/* Execution path of the stage calls: AUTO picks one CTA per molecule with its SCF matrices in
 * shared memory for nao <= 160 and the grid-wide kernels (host-driven SCF loop, products on the
 * whole GPU) above that; CTA / GRID force one (CTA keeps its work matrices in global memory
 * above nao 160 and refuses SCF above nao 1024). */
#define SGB_PATH_AUTO 0
#define SGB_PATH_CTA 1
#define SGB_PATH_GRID 2
int sgb_mol_set_path(sgb_mol *mol, int path);
/* nao (ListAtomicOrbitals::size), nocc (DensityMatrix::NumberOfElectrons/2), integral
 * doubles. */
int sgb_mol_info(const sgb_mol *mol, int *natoms, int *nao, int *nocc, long long *nblocks);
/* Replaces TwoCenterIntegral::ComputeAllTwoCenterIntegral + To_device
 * (twocenterintegral.cpp:229-279, 23-53). */
int sgb_two_center(sgb_ctx *ctx, sgb_mol *mol);
/* Replaces Hcore::ComputeMatrix (hcore.cpp:104-124). */
int sgb_hcore(sgb_ctx *ctx, sgb_mol *mol);
/* Replaces SCFCalculation::AllocSCFData + ComputeSCF (scfcalculation.cpp:29-146) with the
 * energy threshold (hard-coded 5e-3 eV at scfcalculation.cpp:77) and the step cap (100, :74)
 * as arguments.  energies (optional, max_iter+1 doubles) receives E_0 .. E_n_iter. */
int sgb_scf(sgb_ctx *ctx, sgb_mol *mol, double tol, int max_iter, sgb_scf_result *result,
            double *energies);
/* Replaces CoreCoreRepulsion::ComputeRepulsion (corecorerepulsion.cpp:12-41). */
int sgb_core_core(sgb_ctx *ctx, sgb_mol *mol, double *e_cc);
/* Replaces FockMatrix::ComputeMatrix (fockmatrix.cpp:32-53) followed by
 * ElectronicEnergy::ComputeEnergy (electronicenergy.cpp:12-36) for a caller-given packed
 * density P: F = Hcore + G(P) into F (packed, host), E_el into *e_el (may be NULL). */
int sgb_fock(sgb_ctx *ctx, sgb_mol *mol, const double *P, double *F, double *e_el);
/* Replaces ElectronicEnergy::ComputeEnergy (electronicenergy.cpp:12-36): E_el =
 * 1/2 sum_ij P_ij (H_ij + F_ij) over caller-given packed nao x nao matrices, reduced on the
 * device in a fixed order. */
int sgb_electronic_energy(sgb_ctx *ctx, int nao, const double *H, const double *F,
                          const double *P, double *e_el);
/* Copies one of SGB_BLOCKS .. SGB_EIGVEC to host memory (sizes: see sgb_mol_info; packed
 * matrices nao*(nao+1)/2, SGB_EIGVAL nao, SGB_EIGVEC nao*nao).  Replaces reading
 * TwoCenterIntegral::GetValueFromArray / BaseMatrix::matrixHold_ / SCFCalculation::eigenVec. */
int sgb_get(sgb_ctx *ctx, const sgb_mol *mol, int which, double *host, size_t count);

/* ---- many molecules in one launch (batched / persistent path) -------------------------- */
/* nmol molecules, natoms[m] atoms each; Z and xyz concatenated in molecule order. */
int sgb_batch_create(sgb_ctx *ctx, int nmol, const int *natoms, const int *Z, const double *xyz,
                     sgb_batch **out);
int sgb_batch_destroy(sgb_batch *b);
/* Replaces new coordinates for the same molecules (same atom counts and elements): one
 * host->device copy of natoms_total*3 doubles. */
int sgb_batch_set_coordinates(sgb_ctx *ctx, sgb_batch *b, const double *xyz);
/* Integrals, Hcore, SCF and core-core repulsion of every molecule, one persistent launch per
 * size class; one CTA per molecule, nao <= 1024 (larger: SGB_E_UNSUPPORTED, use sgb_scf). */
int sgb_batch_run(sgb_ctx *ctx, sgb_batch *b, double tol, int max_iter);
/* Per-molecule results (any pointer may be NULL).  Blocks until the run has finished. */
int sgb_batch_results(sgb_ctx *ctx, sgb_batch *b, double *e_el, double *e_cc, int *n_iter,
                      int *converged, int *status);
/* One call for a set of molecules from host arrays: create (reusing the context's cached
 * batch when the shapes match), run, read results.  e_tot may be NULL. */
int sgb_run_molecules(sgb_ctx *ctx, int nmol, const int *natoms, const int *Z, const double *xyz,
                      double tol, int max_iter, double *e_el, double *e_cc, int *n_iter,
                      int *converged, int *status);
/* Geometry gradient of the total energy, dE_tot/dxyz in eV/Angstrom (natoms*3 values, the
 * order of xyz), by central differences: the molecule and its 6 natoms copies displaced by
 * +/- step Angstrom along each coordinate run as one batch (one CTA per geometry, nao <= 1024);
 * *e_tot (may be NULL) receives the undisplaced total energy.  The SCF tolerance sets the
 * noise: about tol / step (use tol near 1e-9 eV with step 1e-4 Angstrom).  Any geometry whose
 * SCF stops (SGB_E_EIG, SGB_E_NAN) or reaches max_iter unconverged (SGB_E_NOCONV) fails the
 * call, and grad is then not written.  No counterpart in
 * the reference, whose README lists a geometry optimizer as future work (README.md:110). */
int sgb_gradient(sgb_ctx *ctx, int natoms, const int *Z, const double *xyz, double tol,
                 int max_iter, double step, double *e_tot, double *grad);
/* Kernel launches one sgb_batch_run makes (one persistent launch per occupied size class). */
int sgb_batch_launches(const sgb_batch *b, int *launches);
/* Device-time of the last sgb_batch_run in milliseconds (CUDA events on the context stream). */
int sgb_batch_last_ms(const sgb_batch *b, float *ms);
/* Per-molecule device timestamps (ns, %globaltimer) of the last run: when its CTA started the
 * molecule and when its energies were written.  Latency of molecule m inside the launch:
 * t_end[m] - min(t_begin). */
int sgb_batch_timestamps(sgb_ctx *ctx, sgb_batch *b, unsigned long long *t_begin,
                         unsigned long long *t_end);
/* Stage timers (the reference prints per-step Lapack/Pmat/Fmat/Ener times,
 * scfcalculation.cpp:83-140).  When on, each run records per molecule SGB_STAGE_SLOTS
 * counters: SM cycles of integrals, Hcore, Fock+energy, warm-start product, Jacobi,
 * eigenvalues+sort, density, core-core, purification; then counts: Jacobi sweeps,
 * occupied-virtual eigensolves, full eigensolves, purification products. */
#define SGB_STAGE_SLOTS 13
int sgb_batch_set_profiling(sgb_batch *b, int on);
int sgb_batch_stage_cycles(sgb_ctx *ctx, sgb_batch *b, unsigned long long *cycles);
/* Device pointer of the batch's coordinate buffer (natoms_total*3 doubles) for callers that
 * stage inputs themselves. */
int sgb_batch_device_coordinates(sgb_batch *b, void **dptr);

/* ---- one molecule without any device allocation ----------------------------------------- */
/* No counterpart in the reference.  For callers that may not allocate device memory: code
 * running inside a host framework that owns the GPU's memory through its own pool and forbids
 * other allocations, or code that must not allocate after it has started.  Runs one molecule's
 * whole calculation (integrals, Hcore, SCF to |dE| < tol within max_iter steps, core-core
 * repulsion) on the CURRENT device, on `stream` (a cudaStream_t; NULL = the default stream), and
 * returns when the results are in the host outputs (any output pointer may be NULL).  It calls
 * no cudaMalloc / cudaFree and no allocating library routine: all device scratch is a 1 MiB
 * static array that every GPU which loads this library holds until the process exits.
 * Limit: at most 128 atoms and 128 atomic orbitals (e.g. C32, C20H42); larger molecules are
 * rejected with SGB_E_UNSUPPORTED before any GPU work.  The first call on a device does that
 * device's set-up (loads the MNDO tables, looks up the scratch's device address), so it should
 * come before any stream capture.  Each call is synchronous: it copies its inputs from host
 * memory, and returns only after `stream` has finished the molecule and the results have been
 * copied back.  Every call on a device uses the same scratch, which keeps the previous call's
 * contents: calls whose GPU work overlaps (other streams, other host threads) race and must be
 * serialised by the caller.  The solver follows SGB_DENSITY_SOLVER (see above).  Returns
 * SGB_OK, SGB_E_EIG, SGB_E_NAN, or an error. */
int sgb_scf_noalloc(int natoms, const int *Z, const double *xyz, double tol, int max_iter,
                    void *stream, double *e_el, double *e_cc, int *n_iter, int *converged,
                    int *status);

#ifdef __cplusplus
}
#endif
#endif /* SEMIGPU_B200_H */
