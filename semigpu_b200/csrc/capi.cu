// C ABI of the engine (include/semigpu_b200.h).  One translation unit: the device tables live
// in this TU's constant bank, and every kernel is instantiated here.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/semigpu_b200.h"
#include "batch_scf.cuh"
#include "grid_purify.cuh"
#include "grid_purify32.cuh"
#include "grid_scf.cuh"
#include "layout.h"
#include "mndo_tables.cuh"

using namespace sgb;

namespace {

constexpr int kSmallNmax = 160;  // largest nao whose n x n FP64 matrix fits one CTA's smem

// Size classes of the batched launch, by nao: (upper bound, eigenvector column registers per
// lane, default threads per CTA; smaller molecules take smaller CTAs, several per SM).  Up to
// nao 160 the eigensolver's columns sit in registers and shared memory; the class up to 1024
// streams them from global memory (CR 0).  The last class holds molecules too large for one
// CTA's SCF; only the integral, Hcore, Fock and core-core stages run there (their SCF is the
// grid path of sgb_scf).
struct SizeClass {
  int nmax, cr, threads;
};
constexpr SizeClass kClasses[] = {{32, 2, 128},  {64, 2, 256},   {96, 3, 512},     {128, 4, 512},
                                  {160, 5, 512}, {1024, 0, 512}, {1 << 30, 0, 512}};
constexpr int kNumClasses = 7;
constexpr int kBatchScfMax = 1024;  // one CTA per molecule up to here; the grid path above

// SGB_SOLVER_PURIFY unless the environment sets SGB_DENSITY_SOLVER=jacobi or =mixed.
int default_solver() {
  const char* env = getenv("SGB_DENSITY_SOLVER");
  if (env && strcmp(env, "jacobi") == 0) return SOLVER_JACOBI;
  if (env && strcmp(env, "mixed") == 0) return SOLVER_PURIFY_MIXED;
  return SOLVER_PURIFY;
}

// CTA sizes a class can launch with (launch_class): the streamed class only 512 threads, the
// classes whose columns fit 2 registers per lane also 128.
bool class_threads_ok(int k, int t) {
  if (k < 0 || k >= kNumClasses) return false;
  if (kClasses[k].cr == 0) return t == 512;
  return t == 256 || t == 512 || (t == 128 && kClasses[k].cr == 2);
}

int class_of(int nao) {
  int c = 0;
  while (nao > kClasses[c].nmax) ++c;
  return c;
}
constexpr size_t kAlign = 256;

__global__ void k_ang_to_bohr(const double* __restrict__ xyz, double* __restrict__ pos,
                              int64_t count) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x)
    pos[i] = xyz[i] * kAng2Bohr;
}

}  // namespace

struct sgb_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  size_t budget = 0;
  size_t in_use = 0;
  int num_sms = 0;
  size_t smem_optin = 0;
  std::string err;
  sgb_batch* cached = nullptr;  // reused by sgb_run_molecules
  cudaStream_t aux[kNumClasses] = {};
  cudaEvent_t joined[kNumClasses] = {};
  int class_threads[kNumClasses] = {};
  int solver = SOLVER_PURIFY;  // SGB_SOLVER_*
  int sm_limit = 0;            // batched launches use at most this many SMs' worth of CTAs (0: all)
  int diis = 0;                // DIIS depth of the grid-path SCF (0: off)
  int max_sweeps = 0;          // Jacobi sweeps per eigensolve (0: the path's default)
  long long wait_spins = -1;   // polls of a bounded device wait (< 0: the default bound)
  double damping = 0.0;        // density damping factor (0: off)
  int grid_config = -1;        // tile configuration of the whole-GPU purification (-1: by size)
  // Timing events for batches, created with the context and recycled: cudaEventCreate waits
  // for the kernels running on the device, which would stall a batch built while another
  // context's long launch runs.
  std::vector<cudaEvent_t> events;
  std::mutex events_mutex;
  // optional reusable arena (sgb_ctx_reserve): a batch that fits takes it instead of calling
  // cudaMalloc, and gives it back without cudaFree (which would synchronise the device)
  char* pool = nullptr;
  size_t pool_bytes = 0;
  bool pool_busy = false;
  // Device arenas given back by destroyed batches, molecules and grid workspaces, kept for the
  // next ones: cudaFree synchronises the whole device and cudaMalloc can wait behind running
  // kernels, so create/destroy cycles of similar sizes (one molecule per call) allocate
  // nothing once warm.  Counted in in_use; released when the budget or a failed cudaMalloc
  // needs the room, and with the context.
  std::vector<std::pair<char*, size_t>> spare;
  size_t spare_bytes = 0;
  std::mutex spare_mutex;
  // pinned host buffer for copies between caller memory and the device (upload / download)
  char* staging = nullptr;
  size_t staging_bytes = 0;
  cudaEvent_t staging_ev = nullptr;  // recorded after the last uploads read from it
  bool staging_busy = false;
  // live batches and molecules of this context: sgb_ctx_destroy releases their device memory
  // and detaches them, so destroying one afterwards (a garbage-collected wrapper) frees only
  // its host part and never touches the freed context
  std::vector<sgb_batch*> batches;
  std::vector<sgb_mol*> mols;
};

struct sgb_batch {
  sgb_ctx* ctx = nullptr;
  int nmol = 0;
  int64_t natoms_total = 0;
  int nmax = 0;
  std::vector<MolDesc> desc;
  std::vector<int> order;
  std::vector<int> natoms;
  std::vector<int> Z;
  int class_first[kNumClasses] = {}, class_count[kNumClasses] = {}, class_nmax[kNumClasses] = {};
  char* arena = nullptr;
  size_t bytes = 0;
  bool from_pool = false;
  char* diis = nullptr;  // DIIS history (batched SCF with sgb_ctx_set_diis), on first use
  size_t diis_bytes = 0;
  int diis_depth = 0;
  MolDesc* d_desc = nullptr;
  int* d_order = nullptr;
  int* d_counter = nullptr;
  int8_t* d_slot = nullptr;
  double* d_xyz = nullptr;
  double* d_pos = nullptr;
  int* d_first = nullptr;
  int64_t* d_row_off = nullptr;
  int* d_hb = nullptr;
  double *d_ints = nullptr, *d_H = nullptr, *d_P = nullptr, *d_F = nullptr;
  double *d_V = nullptr, *d_T = nullptr, *d_eig = nullptr, *d_W = nullptr;
  CUtensorMap* d_maps = nullptr;  // work-matrix tensor maps of the molecules above nao 160
  double *d_eel = nullptr, *d_ecc = nullptr;
  int *d_niter = nullptr, *d_conv = nullptr, *d_status = nullptr;
  unsigned long long *d_tb = nullptr, *d_te = nullptr;
  unsigned long long* d_stage = nullptr;
  bool profiling = false;
  double* d_hist = nullptr;
  int hist_stride = 0;
  int64_t n_ints = 0, n_pk = 0, n_sq = 0, n_ao = 0, n_w = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
};

// Device workspace of the grid-wide path (allocated on first use).
struct GridWork {
  char* arena = nullptr;
  size_t bytes = 0;
  double *G = nullptr, *Fprev = nullptr, *wq = nullptr, *dval = nullptr, *partial = nullptr;
  double* X2 = nullptr;  // purification: X and its partner are G and X2 (padded order xnp)
  int xbuf = 0;          // which of G (0) / X2 (1) holds the last purified X
  int xnp = 0;           // its padded order
  unsigned* count = nullptr;  // last-block counter of the fused reductions (0 between uses)
  // DIIS history (grid path, when enabled): depth x (F, error) n x n pairs, and the B matrix
  double* diis = nullptr;
  int diis_cap = 0;
  size_t diis_bytes = 0;
  double* scalars = nullptr;  // [0] E_el, [1] E_cc
  int *occ = nullptr, *vir = nullptr, *flag = nullptr, *result = nullptr;
  unsigned long long* worst = nullptr;
  unsigned* bar = nullptr;  // count, generation
  int* err = nullptr;
};

struct sgb_mol {
  sgb_ctx* ctx = nullptr;
  sgb_batch* b = nullptr;
  bool ints_done = false, hcore_done = false, scf_done = false;
  bool eig_pending = false;  // grid purification: eigenpairs of Fprev computed on first read
  int path = SGB_PATH_AUTO;
  GridWork gw;
};

namespace {

int fail(sgb_ctx* ctx, int code, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return code;
}

int cuda_fail(sgb_ctx* ctx, cudaError_t e, const char* what) {
  return fail(ctx, SGB_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CUDA_TRY(ctx, call)                                  \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// Estimated SCF cost used to order the persistent launch (largest first).
double cost_of(const MolDesc& d) { return (double)d.nao * d.nao * d.nao + 50.0 * d.natoms * d.natoms; }

cudaError_t take_event(sgb_ctx* ctx, cudaEvent_t* ev) {
  {
    std::lock_guard<std::mutex> lock(ctx->events_mutex);
    if (!ctx->events.empty()) {
      *ev = ctx->events.back();
      ctx->events.pop_back();
      return cudaSuccess;
    }
  }
  return cudaEventCreate(ev);
}

void give_event(sgb_ctx* ctx, cudaEvent_t ev) {
  if (!ev) return;
  if (!ctx) {
    cudaEventDestroy(ev);
    return;
  }
  std::lock_guard<std::mutex> lock(ctx->events_mutex);
  ctx->events.push_back(ev);
}

constexpr size_t kSpareMaxBlocks = 16;
constexpr size_t kSpareMaxBytes = size_t(8) << 30;

// Arena sizes: at least 1 MiB, then four sizes per power of two (at most 25 % over the
// request), so the arenas of molecules of similar size are interchangeable.
size_t arena_size_class(size_t bytes) {
  if (bytes <= (size_t(1) << 20)) return size_t(1) << 20;
  const int lg = 63 - __builtin_clzll((unsigned long long)bytes);
  const size_t step = size_t(1) << (lg - 2);
  return (bytes + step - 1) / step * step;
}

// Frees spare arenas, largest first, until at most keep_blocks / keep_bytes remain and
// in_use + need fits the budget.  Caller holds spare_mutex.
void release_spares(sgb_ctx* ctx, size_t keep_blocks, size_t keep_bytes, size_t need = 0) {
  while (!ctx->spare.empty() &&
         (ctx->spare.size() > keep_blocks || ctx->spare_bytes > keep_bytes ||
          (ctx->budget && ctx->in_use + need > ctx->budget))) {
    auto big = std::max_element(ctx->spare.begin(), ctx->spare.end(),
                                [](const std::pair<char*, size_t>& a,
                                   const std::pair<char*, size_t>& b) { return a.second < b.second; });
    cudaFree(big->first);
    ctx->spare_bytes -= big->second;
    ctx->in_use -= big->second;
    ctx->spare.erase(big);
  }
}

// A device arena of at least `bytes`: the best-fitting spare (at most 4x the request), else a
// new cudaMalloc within the budget.  *got = the arena's size (what arena_put takes back).
int arena_get(sgb_ctx* ctx, size_t bytes, const char* what, char** out, size_t* got) {
  std::lock_guard<std::mutex> lock(ctx->spare_mutex);
  int best = -1;
  for (int i = 0; i < (int)ctx->spare.size(); ++i) {
    const size_t sz = ctx->spare[i].second;
    if (sz >= bytes && sz <= 4 * bytes + (size_t(1) << 20) &&
        (best < 0 || sz < ctx->spare[best].second))
      best = i;
  }
  if (best >= 0) {
    *out = ctx->spare[best].first;
    *got = ctx->spare[best].second;
    ctx->spare_bytes -= *got;
    ctx->spare.erase(ctx->spare.begin() + best);
    return SGB_OK;
  }
  const size_t sz = arena_size_class(bytes);
  release_spares(ctx, kSpareMaxBlocks, kSpareMaxBytes, sz);
  if (ctx->budget && ctx->in_use + sz > ctx->budget)
    return fail(ctx, SGB_E_NOMEM, "%s needs %zu bytes; budget %zu, in use %zu", what, sz,
                ctx->budget, ctx->in_use);
  cudaError_t e = cudaMalloc(out, sz);
  if (e != cudaSuccess && !ctx->spare.empty()) {
    cudaGetLastError();
    release_spares(ctx, 0, 0);
    e = cudaMalloc(out, sz);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    return fail(ctx, SGB_E_NOMEM, "cudaMalloc(%zu) for %s: %s", sz, what, cudaGetErrorString(e));
  }
  ctx->in_use += sz;
  *got = sz;
  return SGB_OK;
}

// Takes an arena back once the context's stream (which every launch of the context joins)
// has finished with it.
void arena_put(sgb_ctx* ctx, char* p, size_t bytes) {
  if (!p) return;
  if (!ctx) {
    cudaFree(p);
    return;
  }
  cudaStreamSynchronize(ctx->stream);
  std::lock_guard<std::mutex> lock(ctx->spare_mutex);
  ctx->spare.emplace_back(p, bytes);
  ctx->spare_bytes += bytes;
  release_spares(ctx, kSpareMaxBlocks, kSpareMaxBytes);
}

// ---- host staging ----
// A cudaMemcpyAsync to or from pageable memory is staged by the driver, and such a copy was seen
// to wait behind another host thread's pending pageable copy: a 1 KB read-back held up for the
// 2 s of another context's launch.  The copies between caller memory and the device therefore go
// through the context's own pinned buffer (plain DMA on its stream); memory the caller pinned
// is copied directly.
constexpr size_t kStagingBytes = size_t(8) << 20;

struct HostCopy {
  void* dst;
  const void* src;
  size_t bytes;
};

bool host_pinned(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

size_t staged_bytes(const HostCopy* c, int n) {
  size_t total = 0;
  for (int i = 0; i < n; ++i) total += (c[i].bytes + 15) & ~size_t(15);
  return total;
}

// Host -> device copies on st.  Staged sources are copied into the buffer at once, so the
// caller's memory may be reused on return; the buffer is reused only after these copies ran.
cudaError_t upload(sgb_ctx* ctx, const HostCopy* c, int n, cudaStream_t st) {
  const bool stage = ctx->staging && staged_bytes(c, n) <= ctx->staging_bytes;
  cudaError_t e;
  if (stage && ctx->staging_busy && (e = cudaEventSynchronize(ctx->staging_ev)) != cudaSuccess)
    return e;
  size_t off = 0;
  for (int i = 0; i < n; ++i) {
    if (!c[i].bytes) continue;
    if (stage && !host_pinned(c[i].src)) {
      memcpy(ctx->staging + off, c[i].src, c[i].bytes);
      e = cudaMemcpyAsync(c[i].dst, ctx->staging + off, c[i].bytes, cudaMemcpyHostToDevice, st);
      off += (c[i].bytes + 15) & ~size_t(15);
    } else {
      e = cudaMemcpyAsync(c[i].dst, c[i].src, c[i].bytes, cudaMemcpyHostToDevice, st);
    }
    if (e != cudaSuccess) return e;
  }
  if (off) {
    if ((e = cudaEventRecord(ctx->staging_ev, st)) != cudaSuccess) return e;
    ctx->staging_busy = true;
  }
  return cudaSuccess;
}

// Device -> host copies on st; returns when they have landed in the caller's memory.
cudaError_t download(sgb_ctx* ctx, const HostCopy* c, int n, cudaStream_t st) {
  const bool stage = ctx->staging && staged_bytes(c, n) <= ctx->staging_bytes;
  cudaError_t e;
  if (stage && ctx->staging_busy && (e = cudaEventSynchronize(ctx->staging_ev)) != cudaSuccess)
    return e;
  size_t off = 0;
  std::vector<size_t> at(n, ~size_t(0));
  for (int i = 0; i < n; ++i) {
    if (!c[i].bytes || !c[i].dst) continue;
    if (stage && !host_pinned(c[i].dst)) {
      at[i] = off;
      e = cudaMemcpyAsync(ctx->staging + off, c[i].src, c[i].bytes, cudaMemcpyDeviceToHost, st);
      off += (c[i].bytes + 15) & ~size_t(15);
    } else {
      e = cudaMemcpyAsync(c[i].dst, c[i].src, c[i].bytes, cudaMemcpyDeviceToHost, st);
    }
    if (e != cudaSuccess) return e;
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  ctx->staging_busy = false;
  for (int i = 0; i < n; ++i)
    if (at[i] != ~size_t(0)) memcpy(c[i].dst, ctx->staging + at[i], c[i].bytes);
  return cudaSuccess;
}

void free_batch(sgb_batch* b) {
  if (!b) return;
  if (b->ctx) {
    auto& v = b->ctx->batches;
    v.erase(std::remove(v.begin(), v.end(), b), v.end());
  }
  if (b->arena && b->from_pool) {
    b->ctx->pool_busy = false;
  } else if (b->arena) {
    arena_put(b->ctx, b->arena, b->bytes);
  }
  if (b->diis) arena_put(b->ctx, b->diis, b->diis_bytes);
  give_event(b->ctx, b->ev0);
  give_event(b->ctx, b->ev1);
  delete b;
}

int build_batch(sgb_ctx* ctx, int nmol, const int* natoms, const int* Z, const double* xyz,
                int hist_stride, sgb_batch** out) {
  if (!ctx || !out || nmol <= 0 || !natoms || !Z || !xyz)
    return fail(ctx, SGB_E_ARG, "batch: null pointer or nmol <= 0");
  auto* b = new sgb_batch();
  b->ctx = ctx;
  b->nmol = nmol;
  b->desc.resize(nmol);
  b->natoms.assign(natoms, natoms + nmol);
  int64_t atom0 = 0, blk0 = 0, pk0 = 0, sq0 = 0, ao0 = 0, w0 = 0;
  int nmaps = 0;
  std::vector<int8_t> slot;
  std::vector<int> first, hb;
  std::vector<int64_t> row_off;
  for (int m = 0; m < nmol; ++m) {
    const int na = natoms[m];
    if (na <= 0) { delete b; return fail(ctx, SGB_E_ARG, "molecule %d has %d atoms", m, na); }
    MolDesc& d = b->desc[m];
    d.natoms = na;
    d.atom0 = atom0;
    int nao = 0, nel = 0, nheavy = 0;
    int64_t roff = 0;
    for (int a = 0; a < na; ++a) {
      const int z = Z[atom0 + a];
      const int s = slot_of(z);
      if (s < 0) {
        delete b;
        return fail(ctx, SGB_E_ELEMENT,
                    "molecule %d atom %d: Z=%d has no MNDO parameters (supported: H C N O)", m, a, z);
      }
      slot.push_back((int8_t)s);
      first.push_back(nao);
      hb.push_back(nheavy);
      row_off.push_back(roff);
      // row size of atom a (blocks against atoms 0..a)
      const bool heavy = s != 0;
      const int nh = nheavy + (heavy ? 1 : 0), nl = a + 1 - nh;
      roff += (int64_t)nh * (heavy ? 100 : 10) + (int64_t)nl * (heavy ? 10 : 1);
      nao += heavy ? 4 : 1;
      nel += s == 0 ? 1 : (z - 2);
      nheavy += heavy ? 1 : 0;
      b->Z.push_back(z);
    }
    d.nao = nao;
    d.nocc = nel / 2;
    d.nheavy = nheavy;
    d.nblk = roff;
    d.blk0 = blk0;
    d.pk0 = pk0;
    d.sq0 = sq0;
    d.ao0 = ao0;
    d.w0 = w0;
    d.wmap = -1;
    d.pad_ = 0;
    if (nao > kGsmemMax) {  // Jacobi's G (n x n) or purification's X and Y
      const int64_t need = std::max<int64_t>((int64_t)nao * nao, 2 * (int64_t)purify_doubles(nao));
      w0 += (need + 31) / 32 * 32;
      d.wmap = nmaps++;
    }
    blk0 += (roff + 31) / 32 * 32;
    pk0 += (tri(nao) + 31) / 32 * 32;
    sq0 += ((int64_t)nao * nao + 31) / 32 * 32;
    ao0 += (nao + 31) / 32 * 32;
    atom0 += na;
    b->nmax = std::max(b->nmax, nao);
  }
  b->natoms_total = atom0;
  b->n_ints = blk0; b->n_pk = pk0; b->n_sq = sq0; b->n_ao = ao0; b->n_w = w0;
  b->hist_stride = hist_stride;
  // order: grouped by size class, largest estimated cost first within a class
  b->order.resize(nmol);
  for (int m = 0; m < nmol; ++m) b->order[m] = m;
  std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) {
    const int cx = class_of(b->desc[x].nao), cy = class_of(b->desc[y].nao);
    if (cx != cy) return cx > cy;
    return cost_of(b->desc[x]) > cost_of(b->desc[y]);
  });
  for (int q = 0; q < nmol; ++q) {
    const int c = class_of(b->desc[b->order[q]].nao);
    if (!b->class_count[c]) b->class_first[c] = q;
    ++b->class_count[c];
    b->class_nmax[c] = std::max(b->class_nmax[c], b->desc[b->order[q]].nao);
  }

  // one arena
  const int64_t NA = atom0;
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off = align_up(off + bytes); return o; };
  const size_t o_desc = take(sizeof(MolDesc) * nmol), o_order = take(sizeof(int) * nmol),
               o_counter = take(sizeof(int) * kNumClasses), o_slot = take(NA), o_xyz = take(24 * NA),
               o_pos = take(24 * NA), o_first = take(4 * NA), o_roff = take(8 * NA),
               o_hb = take(4 * NA), o_ints = take(8 * b->n_ints), o_H = take(8 * b->n_pk),
               o_P = take(8 * b->n_pk), o_F = take(8 * b->n_pk), o_V = take(8 * b->n_sq),
               o_T = take(8 * b->n_sq), o_W = take(8 * b->n_w), o_eig = take(8 * b->n_ao),
               o_eel = take(8 * nmol),
               o_ecc = take(8 * nmol), o_nit = take(4 * nmol), o_conv = take(4 * nmol),
               o_stat = take(4 * nmol), o_tb = take(8 * nmol), o_te = take(8 * nmol),
               o_stage = take(8 * (size_t)kStageSlots * nmol),
               o_hist = take(hist_stride > 0 ? 8 * (size_t)hist_stride * nmol : 0),
               o_maps = take(sizeof(CUtensorMap) * kWorkMaps * (size_t)nmaps);
  b->bytes = off;
  cudaError_t e = cudaSuccess;
  if (ctx->pool && !ctx->pool_busy && off <= ctx->pool_bytes) {
    b->arena = ctx->pool;
    b->from_pool = true;
    ctx->pool_busy = true;
  } else {
    const int rc = arena_get(ctx, off, "batch", &b->arena, &b->bytes);
    if (rc) {
      delete b;
      return rc;
    }
  }
  char* base = b->arena;
  b->d_desc = (MolDesc*)(base + o_desc);
  b->d_order = (int*)(base + o_order);
  b->d_counter = (int*)(base + o_counter);
  b->d_slot = (int8_t*)(base + o_slot);
  b->d_xyz = (double*)(base + o_xyz);
  b->d_pos = (double*)(base + o_pos);
  b->d_first = (int*)(base + o_first);
  b->d_row_off = (int64_t*)(base + o_roff);
  b->d_hb = (int*)(base + o_hb);
  b->d_ints = (double*)(base + o_ints);
  b->d_H = (double*)(base + o_H);
  b->d_P = (double*)(base + o_P);
  b->d_F = (double*)(base + o_F);
  b->d_V = (double*)(base + o_V);
  b->d_T = (double*)(base + o_T);
  b->d_W = b->n_w ? (double*)(base + o_W) : nullptr;
  b->d_eig = (double*)(base + o_eig);
  b->d_eel = (double*)(base + o_eel);
  b->d_ecc = (double*)(base + o_ecc);
  b->d_niter = (int*)(base + o_nit);
  b->d_conv = (int*)(base + o_conv);
  b->d_status = (int*)(base + o_stat);
  b->d_tb = (unsigned long long*)(base + o_tb);
  b->d_te = (unsigned long long*)(base + o_te);
  b->d_stage = (unsigned long long*)(base + o_stage);
  b->d_hist = hist_stride > 0 ? (double*)(base + o_hist) : nullptr;
  b->d_maps = nmaps ? (CUtensorMap*)(base + o_maps) : nullptr;
  // tensor maps of the work matrices X and Y of the molecules above nao 160 (n16 x n16, row
  // stride n16 + 8): FP64 X and Y in 64-row boxes of 16 doubles, then for the mixed form the
  // TF32 hi / lo parts of the two sets (set 0 in X's slot, set 1 in Y's; n16 x n16 floats, row
  // stride n16 + 8 floats, 128-row boxes of 32 floats); a molecule whose maps cannot be encoded
  // keeps the purification without TMA
  std::vector<CUtensorMap> maps(kWorkMaps * (size_t)nmaps);
  for (int m = 0; m < nmol && nmaps; ++m) {
    MolDesc& d = b->desc[m];
    if (d.wmap < 0) continue;
    const int n16 = purify_n16(d.nao), ld = purify_ld(d.nao);
    double* X = b->d_W + d.w0;
    double* Y = X + purify_doubles(d.nao);
    CUtensorMap* mp = &maps[kWorkMaps * (size_t)d.wmap];
    bool ok = make_tensor_map_2d(&mp[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, X, n16, n16, ld,
                                 BpCfg::BM, kGpK) &&
              make_tensor_map_2d(&mp[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, Y, n16, n16, ld,
                                 BpCfg::BM, kGpK);
    for (int set = 0; set < 2 && ok; ++set) {
      float* H = reinterpret_cast<float*>(set ? Y : X);
      float* L = H + (int64_t)n16 * ld;
      ok = make_tensor_map_2d(&mp[2 + 2 * set], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, H, n16, n16, ld,
                              kTfBM, kTfK) &&
           make_tensor_map_2d(&mp[3 + 2 * set], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, L, n16, n16, ld,
                              kTfBM, kTfK);
    }
    if (!ok) d.wmap = -1;
  }
  cudaStream_t st = ctx->stream;
  const HostCopy ups[] = {{b->d_desc, b->desc.data(), sizeof(MolDesc) * nmol},
                          {b->d_order, b->order.data(), sizeof(int) * (size_t)nmol},
                          {b->d_slot, slot.data(), (size_t)NA},
                          {b->d_xyz, xyz, 24 * (size_t)NA},
                          {b->d_first, first.data(), 4 * (size_t)NA},
                          {b->d_row_off, row_off.data(), 8 * (size_t)NA},
                          {b->d_hb, hb.data(), 4 * (size_t)NA},
                          {b->d_maps, maps.data(), sizeof(CUtensorMap) * maps.size()}};
  if ((e = upload(ctx, ups, 8, st)) != cudaSuccess ||
      (e = cudaMemsetAsync(b->d_status, 0, 4 * nmol, st)) != cudaSuccess ||
      (e = take_event(ctx, &b->ev0)) != cudaSuccess || (e = take_event(ctx, &b->ev1)) != cudaSuccess) {
    free_batch(b);
    return cuda_fail(ctx, e, "batch upload");
  }
  k_ang_to_bohr<<<std::max<int64_t>(1, std::min<int64_t>((3 * NA + 255) / 256, 1024)), 256, 0, st>>>(
      b->d_xyz, b->d_pos, 3 * NA);
  if ((e = cudaGetLastError()) != cudaSuccess) {
    free_batch(b);
    return cuda_fail(ctx, e, "k_ang_to_bohr");
  }
  ctx->batches.push_back(b);
  *out = b;
  return SGB_OK;
}

// One kernel instantiation per (threads per CTA, eigenvector column registers per lane).
// The dynamic shared memory cap is a per-function attribute shared by every host thread and
// context, so it is raised to the device's opt-in maximum (never to a launch's own size, which
// another thread could lower between its set and its launch), and only once per device:
// setting it waits for the kernels running on the device, which would stall one context's
// launch behind another's long persistent launch.
constexpr int kMaxDevices = 64;

// Raises the kernel's cap on the current device (once); *cap receives it.
template <int NT, int CR, int MX = 0>
cudaError_t kernel_smem_cap(int* cap) {
  auto* k = k_batch_scf<NT, CR, MX>;
  static int max_dynamic[kMaxDevices] = {};  // 0: not set yet on that device
  static std::mutex set_mutex;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(set_mutex);
  if (!max_dynamic[dev]) {
    int optin = 0;
    cudaFuncAttributes fa;
    if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess ||
        (e = cudaFuncGetAttributes(&fa, k)) != cudaSuccess)
      return e;
    const int md = optin - (int)fa.sharedSizeBytes;  // the static part counts against it
    if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, md)) != cudaSuccess)
      return e;
    max_dynamic[dev] = md;
  }
  *cap = max_dynamic[dev];
  return cudaSuccess;
}

// The instances launch_feat<FEAT> can launch.
template <int FEAT>
cudaError_t prepare_feat(int* c) {
  constexpr int D = FEAT & FEAT_DIIS;
  cudaError_t e;
  if ((e = kernel_smem_cap<512, 0, FEAT>(c)) || (e = kernel_smem_cap<128, 2, D>(c)) ||
      (e = kernel_smem_cap<256, 2, D>(c)) || (e = kernel_smem_cap<256, 3, D>(c)) ||
      (e = kernel_smem_cap<256, 4, D>(c)) || (e = kernel_smem_cap<256, 5, D>(c)) ||
      (e = kernel_smem_cap<512, 2, D>(c)) || (e = kernel_smem_cap<512, 3, FEAT>(c)) ||
      (e = kernel_smem_cap<512, 4, FEAT>(c)) || (e = kernel_smem_cap<512, 5, FEAT>(c)))
    return e;
  return cudaSuccess;
}

// Every instantiation, at context creation (before any long launch can be running).
cudaError_t prepare_kernels() {
  int c = 0;
  cudaError_t e;
  if ((e = prepare_feat<0>(&c)) || (e = prepare_feat<FEAT_TENSOR>(&c)) ||
      (e = prepare_feat<FEAT_DIIS>(&c)) || (e = prepare_feat<FEAT_TENSOR | FEAT_DIIS>(&c)))
    return e;
  return cudaSuccess;
}

template <int NT, int CR, int MX = 0>
cudaError_t launch_kernel(int num_sms, const BatchArgs& a, size_t smem, cudaStream_t st) {
  auto* k = k_batch_scf<NT, CR, MX>;
  int cap = 0;
  cudaError_t e = kernel_smem_cap<NT, CR, MX>(&cap);
  if (e != cudaSuccess) return e;
  if (smem > (size_t)cap) return cudaErrorInvalidValue;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NT, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int grid = std::min(a.nmol, per_sm * num_sms);
  k<<<grid, NT, smem, st>>>(a);
  return cudaGetLastError();
}

// FEAT_TENSOR only reaches the 512-thread classes of nao 65-160 (CR 3-5) and the class above
// the shared-memory limit (CR 0); FEAT_DIIS all.
template <int FEAT>
cudaError_t launch_feat(int num_sms, const BatchArgs& a, int cr, int threads, size_t smem,
                        cudaStream_t st) {
  constexpr int D = FEAT & FEAT_DIIS;
  if (cr == 0) return launch_kernel<512, 0, FEAT>(num_sms, a, smem, st);
  if (threads == 128 && cr == 2) return launch_kernel<128, 2, D>(num_sms, a, smem, st);
  if (threads == 512) {
    switch (cr) {
      case 2: return launch_kernel<512, 2, D>(num_sms, a, smem, st);
      case 3: return launch_kernel<512, 3, FEAT>(num_sms, a, smem, st);
      case 4: return launch_kernel<512, 4, FEAT>(num_sms, a, smem, st);
      default: return launch_kernel<512, 5, FEAT>(num_sms, a, smem, st);
    }
  }
  switch (cr) {
    case 2: return launch_kernel<256, 2, D>(num_sms, a, smem, st);
    case 3: return launch_kernel<256, 3, D>(num_sms, a, smem, st);
    case 4: return launch_kernel<256, 4, D>(num_sms, a, smem, st);
    default: return launch_kernel<256, 5, D>(num_sms, a, smem, st);
  }
}

cudaError_t launch_class(int num_sms, const BatchArgs& a, int cr, int threads, size_t smem,
                         cudaStream_t st) {
  const bool tensor = a.solver == SOLVER_PURIFY_MIXED, diis = a.diis && a.diis_depth >= 2;
  if (tensor && diis) return launch_feat<FEAT_TENSOR | FEAT_DIIS>(num_sms, a, cr, threads, smem, st);
  if (tensor) return launch_feat<FEAT_TENSOR>(num_sms, a, cr, threads, smem, st);
  if (diis) return launch_feat<FEAT_DIIS>(num_sms, a, cr, threads, smem, st);
  return launch_feat<0>(num_sms, a, cr, threads, smem, st);
}

// Runs the requested stages over every molecule: one persistent launch per size class, each on
// its own stream so the classes share the GPU, joined back into the context stream.
int launch_stages(sgb_ctx* ctx, sgb_batch* b, int stages, double tol, int max_iter,
                  int sorted_vectors) {
  const bool scf = stages & STAGE_SCF;
  if (scf && b->nmax > kBatchScfMax)
    return fail(ctx, SGB_E_UNSUPPORTED,
                "SCF for nao=%d: one CTA per molecule takes nao <= %d (larger: sgb_scf's grid path)",
                b->nmax, kBatchScfMax);
  BatchArgs a;
  a.mols = b->d_desc;
  a.slot = b->d_slot;
  a.pos = b->d_pos;
  a.first = b->d_first;
  a.row_off = b->d_row_off;
  a.hb = b->d_hb;
  a.ints = b->d_ints;
  a.H = b->d_H; a.P = b->d_P; a.F = b->d_F;
  a.V = b->d_V; a.T = b->d_T; a.eig = b->d_eig; a.W = b->d_W; a.wmaps = b->d_maps;
  a.e_el = b->d_eel; a.e_cc = b->d_ecc;
  a.n_iter = b->d_niter; a.converged = b->d_conv; a.status = b->d_status;
  a.hist = b->d_hist; a.hist_stride = b->hist_stride;
  a.tol = tol;
  a.max_iter = std::min(max_iter, b->hist_stride > 0 ? b->hist_stride - 1 : max_iter);
  a.sorted_vectors = sorted_vectors;
  a.solver = ctx->solver;
  a.stages = stages;
  a.t_begin = b->d_tb;
  a.t_end = b->d_te;
  a.stage_cycles = b->profiling ? b->d_stage : nullptr;
  a.max_sweeps = ctx->max_sweeps > 0 ? ctx->max_sweeps : kBatchJacobiSweeps;
  a.wait_spins = ctx->wait_spins >= 0 ? ctx->wait_spins : kMbarSpins;
  a.damping = ctx->damping;
  if (scf && ctx->diis >= 2) {
    // history of depth F and residual matrices and the last F_in per molecule
    // ((2 depth + 1) n^2) plus its B matrix
    const size_t need =
        8 * ((2 * (size_t)ctx->diis + 1) * (size_t)b->n_sq + (size_t)kDiisB * b->nmol);
    if (b->diis && (b->diis_depth != ctx->diis || b->diis_bytes < need)) {
      arena_put(ctx, b->diis, b->diis_bytes);
      b->diis = nullptr;
    }
    if (!b->diis) {
      if (int rc = arena_get(ctx, need, "DIIS history", &b->diis, &b->diis_bytes)) return rc;
      b->diis_depth = ctx->diis;
    }
    a.diis = reinterpret_cast<double*>(b->diis);
    a.diis_B = a.diis + (2 * (size_t)ctx->diis + 1) * (size_t)b->n_sq;
    a.diis_depth = ctx->diis;
  }
  cudaStream_t st = ctx->stream;
  CUDA_TRY(ctx, cudaMemsetAsync(b->d_counter, 0, sizeof(int) * kNumClasses, st));
  CUDA_TRY(ctx, cudaEventRecord(b->ev0, st));
  int used = 0;
  for (int c = 0; c < kNumClasses; ++c) {
    const int cnt = b->class_count[c];
    if (!cnt) continue;
    BatchArgs ac = a;
    ac.nmol = cnt;
    ac.order = b->d_order + b->class_first[c];
    ac.counter = b->d_counter + c;
    // the Fock and SCF stages keep per-AO work vectors in shared memory; the others need
    // only the reduction slots
    ac.nmax = (stages & (STAGE_SCF | STAGE_FOCK)) ? std::max(1, b->class_nmax[c]) : 1;
    ac.mat_doubles = 0;
    if (stages & (STAGE_SCF | STAGE_FOCK))
      for (int q = 0; q < cnt; ++q)
        ac.mat_doubles = std::max(ac.mat_doubles,
                                  mat_doubles_for(b->desc[b->order[b->class_first[c] + q]].nao));
    size_t smem = (ac.mat_doubles + extra_doubles(ac.nmax)) * sizeof(double);
    // the class above the shared-memory limit purifies through a TMA ring after the rest
    if (kClasses[c].cr == 0 && (stages & STAGE_SCF)) smem += kBpRingBytes;
    cudaStream_t cs = ctx->aux[c];
    CUDA_TRY(ctx, cudaStreamWaitEvent(cs, b->ev0, 0));
    const int sms = ctx->sm_limit > 0 ? std::min(ctx->sm_limit, ctx->num_sms) : ctx->num_sms;
    cudaError_t e = launch_class(sms, ac, kClasses[c].cr, ctx->class_threads[c], smem, cs);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "k_batch_scf launch");
    CUDA_TRY(ctx, cudaEventRecord(ctx->joined[c], cs));
    CUDA_TRY(ctx, cudaStreamWaitEvent(st, ctx->joined[c], 0));
    ++used;
  }
  CUDA_TRY(ctx, cudaEventRecord(b->ev1, st));
  return used ? SGB_OK : fail(ctx, SGB_E_ARG, "empty batch");
}

// ------------------------------------------------------------------------------------------
// Grid-wide path for one molecule

constexpr int kGridThreads = 256;
constexpr int kPartialMax = 4096;
constexpr int kMaxSweeps = 60;

long long barrier_spins(const sgb_ctx* ctx) {
  return ctx->wait_spins >= 0 ? ctx->wait_spins : kBarrierSpins;
}

bool use_grid(const sgb_mol* mol) {
  if (mol->path == SGB_PATH_GRID) return true;
  if (mol->path == SGB_PATH_CTA) return false;
  return mol->b->desc[0].nao > kSmallNmax;
}

MolView mol_view(const sgb_batch* b) {
  const MolDesc& d = b->desc[0];
  MolView v;
  v.natoms = d.natoms; v.nao = d.nao; v.nocc = d.nocc;
  v.slot = b->d_slot; v.pos = b->d_pos; v.first = b->d_first; v.row_off = b->d_row_off;
  v.hb = b->d_hb; v.ints = b->d_ints; v.H = b->d_H; v.P = b->d_P; v.F = b->d_F;
  v.V = b->d_V; v.T = b->d_T; v.eig = b->d_eig;
  return v;
}

int grid_blocks(const sgb_ctx* ctx, int64_t tasks) {
  const int64_t want = (tasks + kGridThreads - 1) / kGridThreads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, std::min<int64_t>(kPartialMax, 8LL * ctx->num_sms)));
}

// Padded order of the purification buffers: a multiple of the largest tile (128), so every
// tile configuration fits the same allocation.
int64_t grid_pad(int64_t n) { return (n + GpLarge::BM - 1) / GpLarge::BM * GpLarge::BM; }

int ensure_grid_work(sgb_ctx* ctx, sgb_mol* mol) {
  GridWork& w = mol->gw;
  if (w.arena) return SGB_OK;
  const int64_t n = mol->b->desc[0].nao;
  const int64_t np = grid_pad(n);  // X and its partner: padded to the largest purify tile
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off = align_up(off + bytes); return o; };
  const size_t oG = take(8 * np * np), oFp = take(8 * n * n), oX2 = take(8 * np * np),
               owq = take(8 * (3 * n + 8)), odv = take(8 * n), opart = take(8 * 2 * kPartialMax),
               osc = take(8 * 16),
               oocc = take(4 * n), ovir = take(4 * n), oflag = take(4), ores = take(16),
               ocount = take(8),
               owst = take(8 * kMaxSweeps), obar = take(8), oerr = take(4);
  if (int rc = arena_get(ctx, off, "grid workspace", &w.arena, &w.bytes)) return rc;
  char* b = w.arena;
  w.G = (double*)(b + oG); w.Fprev = (double*)(b + oFp); w.X2 = (double*)(b + oX2);
  w.wq = (double*)(b + owq);
  w.dval = (double*)(b + odv); w.partial = (double*)(b + opart); w.scalars = (double*)(b + osc);
  w.occ = (int*)(b + oocc); w.vir = (int*)(b + ovir); w.flag = (int*)(b + oflag);
  w.result = (int*)(b + ores); w.worst = (unsigned long long*)(b + owst);
  w.bar = (unsigned*)(b + obar); w.err = (int*)(b + oerr);
  w.count = (unsigned*)(b + ocount);
  CUDA_TRY(ctx, cudaMemsetAsync(w.count, 0, 8, ctx->stream));
  return SGB_OK;
}

void free_grid_work(sgb_ctx* ctx, sgb_mol* mol) {
  if (mol->gw.diis) {
    cudaFree(mol->gw.diis);
    if (ctx) ctx->in_use -= mol->gw.diis_bytes;
  }
  if (mol->gw.arena) {
    arena_put(ctx, mol->gw.arena, mol->gw.bytes);
    mol->gw = GridWork();
  }
}

// F (packed + full into T) and E_el into scalars[0]
int grid_fock(sgb_ctx* ctx, sgb_mol* mol, bool full_matrix) {
  const MolView v = mol_view(mol->b);
  GridWork& w = mol->gw;
  cudaStream_t st = ctx->stream;
  k_grid_pair_density<<<grid_blocks(ctx, (int64_t)v.natoms * 10), kGridThreads, 0, st>>>(v, w.wq);
  const int nb = grid_blocks(ctx, (int64_t)v.natoms * 10 + tri(v.natoms));
  k_grid_fock<<<nb, kGridThreads, 0, st>>>(v, w.wq, full_matrix ? v.T : nullptr, w.partial);
  k_reduce_sum<<<1, 256, 0, st>>>(w.partial, nb, w.scalars);
  CUDA_TRY(ctx, cudaGetLastError());
  return SGB_OK;
}

// One cooperative Jacobi launch; returns sweeps (>0), -1 no convergence, -2 barrier timeout.
int grid_jacobi(sgb_ctx* ctx, sgb_mol* mol, const int* ga, int na, const int* gb, int nb,
                double done_abs, int* sweeps) {
  GridWork& w = mol->gw;
  cudaStream_t st = ctx->stream;
  const int n = mol->b->desc[0].nao;
  CUDA_TRY(ctx, cudaMemsetAsync(w.worst, 0, 8 * kMaxSweeps, st));
  CUDA_TRY(ctx, cudaMemsetAsync(w.bar, 0, 8, st));
  CUDA_TRY(ctx, cudaMemsetAsync(w.err, 0, 4, st));
  GridJacobiArgs a;
  a.n = n; a.G = w.G; a.V = mol->b->d_V;
  a.grp_a = ga; a.na = na; a.grp_b = gb; a.nb = nb;
  a.rot_abs = kJacobiRotAbs; a.done_abs = done_abs;
  a.max_sweeps = ctx->max_sweeps > 0 ? std::min(ctx->max_sweeps, kMaxSweeps) : kMaxSweeps;
  a.worst = w.worst; a.result = w.result;
  a.bar = GridBarrier{w.bar, w.bar + 1, w.err, barrier_spins(ctx), 0u};
  int per_sm = 0;
  CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_grid_jacobi, kGridThreads, 0));
  const int pairs = ga ? na : (n + 1) / 2;
  const int blocks = std::max(1, std::min(per_sm * ctx->num_sms, (pairs * 32 + kGridThreads - 1) / kGridThreads));
  void* args[] = {&a};
  CUDA_TRY(ctx, cudaLaunchCooperativeKernel((void*)k_grid_jacobi, blocks, kGridThreads, args, 0, st));
  int r = 0;
  CUDA_TRY(ctx, cudaMemcpyAsync(&r, w.result, 4, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  *sweeps = r;
  return SGB_OK;
}

// Lanczos-refined bounds (purify.cuh) for the F in T, intersected with the Gershgorin ones
// already in lohi[0..1] (device).  Worth its host round trips only for large n, where one
// product costs milliseconds.
constexpr int kGridLanczosMinN = 1536;

int grid_lanczos_bounds(sgb_ctx* ctx, sgb_mol* mol, double* lohi) {
  const MolView v = mol_view(mol->b);
  GridWork& w = mol->gw;
  cudaStream_t st = ctx->stream;
  const int n = v.nao;
  double* q = w.X2;  // free until the first product
  double* qp = q + n;
  double* wv = qp + n;
  double* sc = w.scalars;
  const int nb = grid_blocks(ctx, n);
  k_lz_start<<<nb, kGridThreads, 0, st>>>(n, q, qp, w.partial);
  k_reduce_sum<<<1, 256, 0, st>>>(w.partial, nb, sc + 6);
  k_lz_scale<<<nb, kGridThreads, 0, st>>>(n, q, sc + 6);
  const int nbr = grid_blocks(ctx, 32LL * n);
  double al[kLanczosSteps], be[kLanczosSteps], beta = 0.0, h[2];
  for (int k = 0; k < kLanczosSteps; ++k) {
    k_lz_matvec<<<nbr, kGridThreads, 0, st>>>(n, v.T, q, qp, beta, wv, w.partial);
    k_reduce_sum<<<1, 256, 0, st>>>(w.partial, nbr, sc + 6);
    k_reduce_sum<<<1, 256, 0, st>>>(w.partial + nbr, nbr, sc + 7);
    CUDA_TRY(ctx, cudaGetLastError());
    CUDA_TRY(ctx, cudaMemcpyAsync(h, sc + 6, 16, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    const double alpha = h[0], nbv = sqrt(std::max(h[1] - alpha * alpha, 0.0));
    al[k] = alpha;
    be[k] = nbv;
    if (!(nbv > 1e-10 * (fabs(alpha) + 1.0))) return SGB_OK;  // invariant subspace: keep Gershgorin
    k_lz_update<<<nb, kGridThreads, 0, st>>>(n, q, qp, wv, alpha, 1.0 / nbv);
    beta = nbv;
  }
  double g[2];
  CUDA_TRY(ctx, cudaMemcpyAsync(g, lohi, 16, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  double llo, lhi;
  lanczos_bounds<kLanczosSteps>(al, be, be[kLanczosSteps - 1], llo, lhi);
  if (llo == llo && lhi == lhi) {
    g[0] = std::max(g[0], llo);
    g[1] = std::min(g[1], lhi);
    CUDA_TRY(ctx, cudaMemcpyAsync(lohi, g, 16, cudaMemcpyHostToDevice, st));
  }
  return SGB_OK;
}

// Tile configuration of the device purification loop for order n: the largest tile that
// still gives every SM work (two tiles per SM for the 128 x 128 tile, one for 64 x 64).
// The tile configurations of the whole-GPU FP64 purification (sgb_grid_configs): tile rows,
// warps, k-blocks per ring stage, stages.
struct GridConfigInfo {
  int bm, warps, kb, stages;
};
constexpr GridConfigInfo kGridConfigs[] = {
    {GpLarge::BM, GpLarge::WARPS, GpLarge::KB, GpLarge::STAGES},
    {GpLargeAlt1::BM, GpLargeAlt1::WARPS, GpLargeAlt1::KB, GpLargeAlt1::STAGES},
    {GpLargeAlt2::BM, GpLargeAlt2::WARPS, GpLargeAlt2::KB, GpLargeAlt2::STAGES},
    {GpMid::BM, GpMid::WARPS, GpMid::KB, GpMid::STAGES},
    {GpSmall::BM, GpSmall::WARPS, GpSmall::KB, GpSmall::STAGES}};
constexpr int kNumGridConfigs = 5;

// Configuration index for order n: the context's choice, else the largest tile that still gives
// every SM work (two tiles per SM for the 128 x 128 tile, one for 64 x 64).
int gp_config(const sgb_ctx* ctx, int n) {
  if (ctx->grid_config >= 0) return ctx->grid_config;
  auto tiles = [](int n, int bm) { const int64_t t = (n + bm - 1) / bm; return t * (t + 1) / 2; };
  if (tiles(n, GpLarge::BM) >= 2LL * ctx->num_sms) return 0;
  if (tiles(n, GpMid::BM) >= ctx->num_sms) return 3;
  return 4;
}


// Dynamic shared memory cap of each configuration, once per device (cudaFuncSetAttribute
// waits for running kernels, so this runs at context creation).
template <class C>
cudaError_t gp_prepare() {
  static bool done[kMaxDevices] = {};
  static std::mutex m;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(m);
  if (!done[dev]) {
    e = cudaFuncSetAttribute(k_grid_purify<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)C::SMEM);
    if (e != cudaSuccess) return e;
    done[dev] = true;
  }
  return cudaSuccess;
}

cudaError_t prepare_grid_purify32() {
  static bool done[kMaxDevices] = {};
  static std::mutex m;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(m);
  if (!done[dev]) {
    e = cudaFuncSetAttribute(k_grid_purify32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kTfSmem);
    if (e != cudaSuccess) return e;
    done[dev] = true;
  }
  return cudaSuccess;
}

cudaError_t prepare_grid_purify() {
  cudaError_t e;
  if ((e = prepare_grid_purify32())) return e;
  if ((e = gp_prepare<GpLarge>()) || (e = gp_prepare<GpMid>()) || (e = gp_prepare<GpSmall>()) ||
      (e = gp_prepare<GpLargeAlt1>()) || (e = gp_prepare<GpLargeAlt2>()))
    return e;
  return cudaSuccess;
}

// One cooperative launch of the device purification loop on X_0 in buffer 0 (padded order
// np, sums at t0); *products and *xbuf from its result.
template <class C>
int gp_launch(sgb_ctx* ctx, sgb_mol* mol, int np, int it0, bool swap, bool mixed, int* products,
              double** xout) {
  GridWork& w = mol->gw;
  cudaStream_t st = ctx->stream;
  const int nocc = mol->b->desc[0].nocc;
  CUtensorMap maps[2];
  double* bufs[2] = {swap ? w.X2 : w.G, swap ? w.G : w.X2};  // X_0 in bufs[0]
  for (int k = 0; k < 2; ++k)
    if (!make_tensor_map_2d(&maps[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, bufs[k], np, np, np,
                            C::BM, kGpK))
      return fail(ctx, SGB_E_CUDA, "tensor map of the purification buffers (np = %d)", np);
  CUDA_TRY(ctx, gp_prepare<C>());
  int per_sm = 0;
  CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_grid_purify<C>,
                                                              C::THREADS, C::SMEM));
  if (per_sm < 1) return fail(ctx, SGB_E_CUDA, "purification kernel does not fit an SM");
  const int nt = np / C::BM;
  const int grid = (int)std::min<int64_t>((int64_t)nt * (nt + 1) / 2,
                                          std::min<int64_t>((int64_t)per_sm * ctx->num_sms,
                                                            kPartialMax / 4));
  CUDA_TRY(ctx, cudaMemsetAsync(w.bar, 0, 8, st));
  CUDA_TRY(ctx, cudaMemsetAsync(w.err, 0, 4, st));
  GridPurifyArgs a;
  a.np = np;
  a.nocc = nocc;
  a.buf[0] = bufs[0];
  a.buf[1] = bufs[1];
  a.partial = w.partial;
  a.t0 = w.scalars + 4;
  a.result = w.result;
  a.bar = GridBarrier{w.bar, w.bar + 1, w.err, barrier_spins(ctx), 0u};
  a.spins = ctx->wait_spins >= 0 ? ctx->wait_spins : kMbarSpins;
  a.it0 = it0;
  a.mixed_finish = mixed ? 1 : 0;
  void* args[] = {&maps[0], &maps[1], &a};
  CUDA_TRY(ctx, cudaLaunchCooperativeKernel((void*)k_grid_purify<C>, grid, C::THREADS, args,
                                            C::SMEM, st));
  int r[2] = {-1, 0};
  CUDA_TRY(ctx, cudaMemcpyAsync(r, w.result, 8, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  if (r[0] == -2) return fail(ctx, SGB_E_CUDA, "a bounded wait of the purification loop gave up");
  *products = r[0];
  *xout = bufs[r[1] & 1];
  return SGB_OK;
}

// The FP32 phase of the mixed form on the tensor cores (grid_purify32.cuh), from X_0 split into
// set 0 (G); *products = products done when tr(X - X^2) fell below the switch point (or -1),
// *set = the set (0: G, 1: X2) holding X.
int gp32_launch(sgb_ctx* ctx, sgb_mol* mol, int np, int* products, int* set) {
  GridWork& w = mol->gw;
  cudaStream_t st = ctx->stream;
  float* H[2] = {reinterpret_cast<float*>(w.G), reinterpret_cast<float*>(w.X2)};
  const int64_t nn = (int64_t)np * np;
  float* L[2] = {H[0] + nn, H[1] + nn};
  CUtensorMap maps[4];
  for (int k = 0; k < 2; ++k)
    if (!make_tensor_map_2d(&maps[2 * k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, H[k], np, np, np,
                            kTfBM, kTfK) ||
        !make_tensor_map_2d(&maps[2 * k + 1], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, L[k], np, np, np,
                            kTfBM, kTfK))
      return fail(ctx, SGB_E_CUDA, "tensor maps of the FP32 purification buffers (np = %d)", np);
  CUDA_TRY(ctx, prepare_grid_purify32());
  int per_sm = 0;
  CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_grid_purify32,
                                                              kTfThreads, kTfSmem));
  if (per_sm < 1) return fail(ctx, SGB_E_CUDA, "FP32 purification kernel does not fit an SM");
  const int nt = np / kTfBM;
  const int grid = (int)std::min<int64_t>((int64_t)nt * (nt + 1) / 2,
                                          std::min<int64_t>((int64_t)per_sm * ctx->num_sms,
                                                            kPartialMax / 4));
  CUDA_TRY(ctx, cudaMemsetAsync(w.bar, 0, 8, st));
  CUDA_TRY(ctx, cudaMemsetAsync(w.err, 0, 4, st));
  GridPurify32Args a;
  a.np = np;
  a.nocc = mol->b->desc[0].nocc;
  a.hi[0] = H[0]; a.hi[1] = H[1];
  a.lo[0] = L[0]; a.lo[1] = L[1];
  a.partial = w.partial;
  a.t0 = w.scalars + 4;
  a.result = w.result;
  a.bar = GridBarrier{w.bar, w.bar + 1, w.err, barrier_spins(ctx), 0u};
  a.spins = ctx->wait_spins >= 0 ? ctx->wait_spins : kMbarSpins;
  a.switch_at = kPurifyMixedSwitch;
  void* args[] = {&maps[0], &maps[1], &maps[2], &maps[3], &a};
  CUDA_TRY(ctx, cudaLaunchCooperativeKernel((void*)k_grid_purify32, grid, kTfThreads, args,
                                            kTfSmem, st));
  int r[2] = {-1, 0};
  CUDA_TRY(ctx, cudaMemcpyAsync(r, w.result, 8, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  if (r[0] == -2)
    return fail(ctx, SGB_E_CUDA, "a bounded wait of the FP32 purification loop gave up");
  *products = r[0];
  *set = r[1] & 1;
  return SGB_OK;
}

// P (packed) from the full F in T by purification (the recursion and limits of purify.cuh);
// *products = number of products, or -1 when it did not converge (the caller diagonalises).
// The FP64 recursion runs on the device in one launch (grid_purify.cuh).  mixed: X and the
// products in FP32 (SSYRK) while tr(X - X^2) >= kPurifyMixedSwitch, then X is widened to FP64
// and the device loop finishes with FP64 products, so the result carries FP64 idempotency; the
// FP32 phase only perturbs the occupied subspace at the 1e-7 level, which enters the energy at
// second order.
int grid_purify(sgb_ctx* ctx, sgb_mol* mol, bool mixed, int* products) {
  const MolView v = mol_view(mol->b);
  GridWork& w = mol->gw;
  cudaStream_t st = ctx->stream;
  const int n = v.nao;
  double* sc = w.scalars;  // [2] lo, [3] hi, [4] tr X, [5] ||X||^2
  const int nbr = grid_blocks(ctx, 32LL * n);
  k_pur_bounds<<<nbr, kGridThreads, 0, st>>>(n, v.T, w.partial);
  k_pur_bounds_reduce<<<1, 32, 0, st>>>(w.partial, nbr, sc + 2);
  if (n >= kGridLanczosMinN) {
    int rc = grid_lanczos_bounds(ctx, mol, sc + 2);
    if (rc) return rc;
  }
  const int cfg = gp_config(ctx, n);
  const int bm = kGridConfigs[cfg].bm;
  const int np = (n + bm - 1) / bm * bm;
  const int nbp = grid_blocks(ctx, (int64_t)np * np);
  *products = -1;
  int it0 = 0, rc;
  bool swap = false;  // X_0 of the FP64 loop in X2 instead of G
  // the tensor-core phase works in 128 x 128 tiles: below one tile per SM (about 2000 AOs) it
  // would leave most SMs idle, and the FP64 loop (smaller tiles) is faster; the mixed form then
  // keeps only its FP64 exit
  const int64_t nt128 = ((int64_t)n + kTfBM - 1) / kTfBM;
  if (mixed && nt128 * (nt128 + 1) / 2 >= ctx->num_sms) {
    // FP32 phase on the tensor cores (TF32 x 3) from X_0 split into hi / lo in G, then X widened
    // into whichever of G / X2 does not hold it, where the FP64 loop continues
    const int np32 = (int)grid_pad(n);
    float* H0 = reinterpret_cast<float*>(w.G);
    k_gp_init32<<<grid_blocks(ctx, (int64_t)np32 * np32), kGridThreads, 0, st>>>(
        n, np32, v.T, sc + 2, H0, H0 + (int64_t)np32 * np32, w.partial, w.count, sc + 4);
    CUDA_TRY(ctx, cudaGetLastError());
    int set = 0;
    if ((rc = gp32_launch(ctx, mol, np32, &it0, &set))) return rc;
    if (it0 < 0) return SGB_OK;  // not finite / no convergence: the caller diagonalises
    const float* Hs = reinterpret_cast<const float*>(set ? w.X2 : w.G);
    const float* Ls = Hs + (int64_t)np32 * np32;
    swap = set == 0;
    k_gp_widen_split<<<nbp, kGridThreads, 0, st>>>(n, np32, Hs, Ls, np, swap ? w.X2 : w.G,
                                                    w.partial, w.count, sc + 4);
  } else {
    k_gp_init<<<nbp, kGridThreads, 0, st>>>(n, np, v.T, sc + 2, w.G, w.partial, w.count, sc + 4);
  }
  CUDA_TRY(ctx, cudaGetLastError());
  int prod = -1;
  double* Xf = nullptr;
  switch (cfg) {
    case 0: rc = gp_launch<GpLarge>(ctx, mol, np, it0, swap, mixed, &prod, &Xf); break;
    case 1: rc = gp_launch<GpLargeAlt1>(ctx, mol, np, it0, swap, mixed, &prod, &Xf); break;
    case 2: rc = gp_launch<GpLargeAlt2>(ctx, mol, np, it0, swap, mixed, &prod, &Xf); break;
    case 3: rc = gp_launch<GpMid>(ctx, mol, np, it0, swap, mixed, &prod, &Xf); break;
    default: rc = gp_launch<GpSmall>(ctx, mol, np, it0, swap, mixed, &prod, &Xf); break;
  }
  if (rc) return rc;
  if (prod >= 0) {
    k_gp_density<<<grid_blocks(ctx, tri(n)), kGridThreads, 0, st>>>(n, np, Xf, v.P, ctx->damping);
    CUDA_TRY(ctx, cudaGetLastError());
    w.xbuf = Xf == w.X2 ? 1 : 0;
    w.xnp = np;
    *products = prod;
  }
  return SGB_OK;
}

// Eigenpairs of the F saved in Fprev (the last one that produced a density), fully
// diagonalised from scratch, sorted ascending into eig / T.
int grid_eigenpairs(sgb_ctx* ctx, sgb_mol* mol) {
  const MolView v = mol_view(mol->b);
  GridWork& w = mol->gw;
  cudaStream_t st = ctx->stream;
  const int n = v.nao;
  k_grid_identity<<<grid_blocks(ctx, (int64_t)n * n), kGridThreads, 0, st>>>(n, mol->b->d_V, w.G, w.Fprev);
  CUDA_TRY(ctx, cudaGetLastError());
  int sw = 0, rc;
  if ((rc = grid_jacobi(ctx, mol, nullptr, 0, nullptr, 0, kJacobiDoneAbs, &sw))) return rc;
  if (sw == -2) return fail(ctx, SGB_E_CUDA, "grid barrier timed out in the Jacobi eigensolver");
  if (sw < 0) return fail(ctx, SGB_E_EIG, "eigenpairs: Jacobi did not converge");
  k_grid_rayleigh<<<grid_blocks(ctx, 32LL * n), kGridThreads, 0, st>>>(n, w.G, mol->b->d_V, w.dval);
  k_grid_sorted_output<<<grid_blocks(ctx, n), kGridThreads, 0, st>>>(n, w.dval, mol->b->d_V, v.eig, v.T);
  CUDA_TRY(ctx, cudaGetLastError());
  mol->eig_pending = false;
  return SGB_OK;
}

// Pulay DIIS for the grid path (optional; changes the SCF trajectory, so off by default).
// After the Fock build of step k, with X = P_k / 2 still in G: store F_k and e_k = F_k P_k -
// P_k F_k, extend B_ij = <e_i, e_j>, solve [B 1; 1^T 0][c; l] = [0; 1] on the host and write
// F = sum c_i F_i into T for the next density.  The reported energy stays that of F_k.
struct DiisState {
  int depth = 0, count = 0, next = 0;
  double B[8][8] = {};
};

int diis_step(sgb_ctx* ctx, sgb_mol* mol, DiisState& ds) {
  const MolView v = mol_view(mol->b);
  GridWork& w = mol->gw;
  cudaStream_t st = ctx->stream;
  const int n = v.nao, depth = ds.depth;
  const int64_t nn = (int64_t)n * n;
  if (w.diis_cap < depth) {
    if (w.diis) {
      cudaFree(w.diis);
      ctx->in_use -= w.diis_bytes;
      w.diis = nullptr;
    }
    const size_t bytes = 2 * (size_t)depth * nn * 8;
    if (ctx->budget && ctx->in_use + bytes > ctx->budget)
      return fail(ctx, SGB_E_NOMEM, "DIIS history needs %zu bytes over the budget", bytes);
    if (cudaMalloc(&w.diis, bytes) != cudaSuccess) return fail(ctx, SGB_E_NOMEM, "DIIS history");
    ctx->in_use += bytes;
    w.diis_bytes = bytes;
    w.diis_cap = depth;
  }
  double* Fh = w.diis;               // depth F matrices
  double* Eh = w.diis + depth * nn;  // depth error matrices
  const int slot = ds.next;
  CUDA_TRY(ctx, cudaMemcpyAsync(Fh + slot * nn, v.T, 8 * nn, cudaMemcpyDeviceToDevice, st));
  // C = F X (X = P / 2, symmetric) and e = C - C^T: the commutator up to the factor 2, to which
  // the DIIS coefficients are insensitive.  The purified X (padded) is unpadded into the free
  // buffer, C overwrites X (P was already written from it).
  const int nb = grid_blocks(ctx, nn);
  double* Xp = w.xbuf ? w.X2 : w.G;
  double* Xu = w.xbuf ? w.G : w.X2;
  k_gp_unpad<<<nb, kGridThreads, 0, st>>>(n, w.xnp, Xp, Xu);
  const dim3 gemm_grid((n + kGemmTile - 1) / kGemmTile, (n + kGemmTile - 1) / kGemmTile);
  k_grid_gemm<<<gemm_grid, 256, 0, st>>>(n, v.T, Xu, Xp);
  k_commutator<<<nb, kGridThreads, 0, st>>>(n, Xp, Eh + slot * nn);
  ds.count = std::min(ds.count + 1, depth);
  ds.next = (slot + 1) % depth;
  for (int j = 0; j < ds.count; ++j) {
    k_dot<<<nb, kGridThreads, 0, st>>>(nn, Eh + slot * nn, Eh + j * nn, w.partial);
    k_reduce_sum<<<1, 256, 0, st>>>(w.partial, nb, w.scalars + 8 + j);
  }
  CUDA_TRY(ctx, cudaGetLastError());
  double row[8];
  CUDA_TRY(ctx, cudaMemcpyAsync(row, w.scalars + 8, 8 * ds.count, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  for (int j = 0; j < ds.count; ++j) ds.B[slot][j] = ds.B[j][slot] = row[j];
  const int m = ds.count;
  if (m < 2) return SGB_OK;
  // [B 1; 1 0] c = [0; 1], Gaussian elimination with partial pivoting (m <= 8), scaled by
  // the largest diagonal entry
  double scale = 0.0;
  for (int i = 0; i < m; ++i) scale = std::max(scale, ds.B[i][i]);
  if (!(scale > 0.0)) return SGB_OK;
  double A[9][10] = {};
  for (int i = 0; i < m; ++i) {
    for (int j = 0; j < m; ++j) A[i][j] = ds.B[i][j] / scale;
    A[i][m] = A[m][i] = 1.0;
  }
  A[m][m + 1] = 1.0;
  for (int c = 0; c <= m; ++c) {
    int piv = c;
    for (int r = c + 1; r <= m; ++r)
      if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
    if (!(fabs(A[piv][c]) > 1e-14)) return SGB_OK;  // singular: keep F_k
    for (int k = 0; k <= m + 1; ++k) std::swap(A[c][k], A[piv][k]);
    for (int r = 0; r <= m; ++r) {
      if (r == c) continue;
      const double f = A[r][c] / A[c][c];
      for (int k = c; k <= m + 1; ++k) A[r][k] -= f * A[c][k];
    }
  }
  LinComb lc;
  lc.m = m;
  for (int i = 0; i < m; ++i) {
    lc.src[i] = Fh + i * nn;
    lc.c[i] = A[i][m + 1] / A[i][i];
    if (!(fabs(lc.c[i]) < 1e6)) return SGB_OK;
  }
  k_lincomb<<<nb, kGridThreads, 0, st>>>(nn, lc, v.T);
  CUDA_TRY(ctx, cudaGetLastError());
  return SGB_OK;
}

int scf_grid(sgb_ctx* ctx, sgb_mol* mol, double tol, int max_iter, sgb_scf_result* res,
             double* energies) {
  int rc = ensure_grid_work(ctx, mol);
  if (rc) return rc;
  sgb_batch* b = mol->b;
  const MolView v = mol_view(b);
  GridWork& w = mol->gw;
  cudaStream_t st = ctx->stream;
  const int n = v.nao, nocc = v.nocc, nvir = n - nocc;
  const int64_t nn = (int64_t)n * n;
  k_grid_guess<<<grid_blocks(ctx, tri(n)), kGridThreads, 0, st>>>(v);
  k_grid_guess_diag<<<grid_blocks(ctx, v.natoms), kGridThreads, 0, st>>>(v);
  if ((rc = grid_fock(ctx, mol, true))) return rc;
  double E = 0.0;
  CUDA_TRY(ctx, cudaMemcpyAsync(&E, w.scalars, 8, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  std::vector<double> hist(1, E);
  int steps = 0, conv = 0, status = SGB_OK;
  if (E != E) status = SGB_E_NAN;  // non-finite input (e.g. a NaN coordinate): no SCF step
  const dim3 gemm_grid((n + kGemmTile - 1) / kGemmTile, (n + kGemmTile - 1) / kGemmTile);
  const bool purify = ctx->solver != SOLVER_JACOBI;
  mol->eig_pending = false;
  DiisState ds;
  ds.depth = purify ? ctx->diis : 0;
  while (status == SGB_OK && !conv && steps < max_iter) {
    const bool cold = steps == 0 || purify;
    bool have_p = false;  // P written by purification; a Jacobi eigensolve only if it failed
    if (purify) {
      int prod = -1;
      if ((rc = grid_purify(ctx, mol, ctx->solver == SOLVER_PURIFY_MIXED, &prod))) return rc;
      have_p = prod >= 0;
    }
    if (!have_p) {
      if (cold)
        k_grid_identity<<<grid_blocks(ctx, nn), kGridThreads, 0, st>>>(n, b->d_V, w.G, v.T);
      else
        k_grid_gemm<<<gemm_grid, 256, 0, st>>>(n, v.T, b->d_V, w.G);
      CUDA_TRY(ctx, cudaGetLastError());
      bool full = cold || steps < kFullJacobiSteps || nocc == 0 || nvir == 0;
      int sw = 0;
      if (!full) {
        k_grid_rayleigh<<<grid_blocks(ctx, 32LL * n), kGridThreads, 0, st>>>(n, w.G, b->d_V, w.dval);
        k_grid_split<<<grid_blocks(ctx, n), kGridThreads, 0, st>>>(n, nocc, w.dval, w.occ, w.vir);
        const bool o_small = nocc <= nvir;
        if ((rc = grid_jacobi(ctx, mol, o_small ? w.occ : w.vir, o_small ? nocc : nvir,
                              o_small ? w.vir : w.occ, o_small ? nvir : nocc, kJacobiDoneGapped, &sw)))
          return rc;
        if (sw > 0) {
          k_grid_rayleigh<<<grid_blocks(ctx, 32LL * n), kGridThreads, 0, st>>>(n, w.G, b->d_V, w.dval);
          k_grid_crossing<<<1, 256, 0, st>>>(nocc, nvir, w.dval, w.occ, w.vir, kCrossMargin, w.flag);
          int cross = 0;
          CUDA_TRY(ctx, cudaMemcpyAsync(&cross, w.flag, 4, cudaMemcpyDeviceToHost, st));
          CUDA_TRY(ctx, cudaStreamSynchronize(st));
          full = cross != 0;
        }
      }
      if (full) {
        if ((rc = grid_jacobi(ctx, mol, nullptr, 0, nullptr, 0, kJacobiDoneAbs, &sw))) return rc;
        if (sw > 0) {
          k_grid_rayleigh<<<grid_blocks(ctx, 32LL * n), kGridThreads, 0, st>>>(n, w.G, b->d_V, w.dval);
          k_grid_split<<<grid_blocks(ctx, n), kGridThreads, 0, st>>>(n, nocc, w.dval, w.occ, w.vir);
        }
      }
      if (sw == -2) return fail(ctx, SGB_E_CUDA, "grid barrier timed out in the Jacobi eigensolver");
      if (sw < 0) { status = SGB_E_EIG; break; }
      if (nocc > 0) {
        const int tiles = (n + 3) / 4;
        k_grid_density<<<grid_blocks(ctx, (int64_t)tiles * (tiles + 1) / 2), kGridThreads, 0, st>>>(
            n, nocc, b->d_V, w.occ, v.P, ctx->damping);
      } else {
        CUDA_TRY(ctx, cudaMemsetAsync(v.P, 0, 8 * tri(n), st));
      }
    }
    // keep the F that produced this density: the final eigenpairs are reported for it
    CUDA_TRY(ctx, cudaMemcpyAsync(w.Fprev, v.T, 8 * nn, cudaMemcpyDeviceToDevice, st));
    if ((rc = grid_fock(ctx, mol, true))) return rc;
    const double Eold = E;
    CUDA_TRY(ctx, cudaMemcpyAsync(&E, w.scalars, 8, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    ++steps;
    hist.push_back(E);
    if (E != E) { status = SGB_E_NAN; break; }
    conv = fabs(Eold - E) < tol;
    if (!conv && ds.depth > 0 && have_p && (rc = diis_step(ctx, mol, ds))) return rc;
  }
  // eigenpairs of the last eigensolve's F, fully diagonalised (the loop may have rotated only
  // occupied-virtual pairs), sorted ascending into eig / T; after purification they are
  // computed when first read (sgb_get)
  if (steps > 0 && status == SGB_OK && purify) {
    mol->eig_pending = true;
  } else if (steps > 0 && status == SGB_OK) {
    k_grid_gemm<<<gemm_grid, 256, 0, st>>>(n, w.Fprev, b->d_V, w.G);
    int sw = 0;
    if ((rc = grid_jacobi(ctx, mol, nullptr, 0, nullptr, 0, kJacobiDoneAbs, &sw))) return rc;
    if (sw < 0) status = SGB_E_EIG;
    k_grid_rayleigh<<<grid_blocks(ctx, 32LL * n), kGridThreads, 0, st>>>(n, w.G, b->d_V, w.dval);
    k_grid_sorted_output<<<grid_blocks(ctx, n), kGridThreads, 0, st>>>(n, w.dval, b->d_V, v.eig, v.T);
    CUDA_TRY(ctx, cudaGetLastError());
  }
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  if (energies) std::copy(hist.begin(), hist.end(), energies);
  if (res) {
    res->e_el = E;
    res->n_iter = steps;
    res->converged = conv;
    res->status = status;
  }
  return status;
}

// ------------------------------------------------------------------------------------------
// Allocation-free single-molecule run (sgb_scf_noalloc).  All of its device scratch -- the
// molecule descriptor, atom arrays, integral blocks, Hcore / P / F, the two n x n matrices and
// the results -- is carved out of one file-scope array that exists for as long as the library
// is loaded.  Host code never touches g_noalloc_scratch by name: its device address comes from
// cudaGetSymbolAddress, fetched once per device.
constexpr int kNoAllocMaxNao = 128;
constexpr int kNoAllocMaxAtoms = 128;
constexpr size_t kNoAllocScratchBytes = size_t(1) << 20;  // 1 MiB per GPU
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct NoAllocDevice {
  bool ready = false;
  unsigned char* scratch = nullptr;
  int num_sms = 0;
};
NoAllocDevice g_noalloc[kNoAllocMaxDevices];
std::mutex g_noalloc_mutex;

// Everything the host writes before a run, staged in one contiguous block (one copy).
struct NoAllocHeader {
  MolDesc desc;
  int order;
  int counter[kNumClasses];
  int8_t slot[kNoAllocMaxAtoms];
  int first[kNoAllocMaxAtoms];
  int hb[kNoAllocMaxAtoms];
  int64_t row_off[kNoAllocMaxAtoms];
  double xyz[3 * kNoAllocMaxAtoms];
};

struct NoAllocResults {
  double e_el, e_cc;
  int n_iter, converged, status, pad;
};

}  // namespace

// ============================================================================================
extern "C" {

const char* sgb_status_string(int s) {
  switch (s) {
    case SGB_OK: return "ok";
    case SGB_E_ARG: return "invalid argument";
    case SGB_E_ELEMENT: return "element without MNDO parameters";
    case SGB_E_CUDA: return "CUDA error";
    case SGB_E_NOMEM: return "out of device memory or over budget";
    case SGB_E_STATE: return "stage called out of order";
    case SGB_E_UNSUPPORTED: return "unsupported size";
    case SGB_E_EIG: return "eigensolver did not converge";
    case SGB_E_NAN: return "non-finite energy";
    case SGB_E_NOCONV: return "SCF did not converge within max_iter";
    default: return "unknown status";
  }
}

const char* sgb_last_error(const sgb_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int sgb_heat_of_formation(int natoms, const int* Z, double e_tot, double* dhf) {
  if (natoms <= 0 || !Z || !dhf) return SGB_E_ARG;
  constexpr double kEvToKcal = 23.060548;  // kcal/mol per eV (CODATA 2018)
  double eisol = 0.0, heat = 0.0;
  for (int a = 0; a < natoms; ++a) {
    double v[SGB_PARAM_COUNT];
    if (sgb_mndo_parameters(Z[a], v) != SGB_OK) return SGB_E_ELEMENT;
    eisol += v[SGB_P_EISOL];
    heat += v[SGB_P_HEAT];
  }
  *dhf = (e_tot - eisol) * kEvToKcal + heat;
  return SGB_OK;
}

int sgb_mndo_parameters(int Z, double* v) {
  const int s = slot_of(Z);
  if (s < 0 || !v) return SGB_E_ELEMENT;
  // exponent, heat of formation of the atom and its computed total energy: parameters the
  // reference stores but its SCF path does not use (MNDO_parameters.cpp:47-122)
  static const double zs[4] = {1.3319670, 1.7875370, 2.25561400, 2.69990500};
  static const double heat[4] = {52.102, 170.89, 113.00000000, 59.55900000};
  static const double eisol[4] = {-11.9062760, -120.500606, -202.56620100, -317.86850600};
  const ElemParams& e = kElemHost[s];
  const double vals[SGB_PARAM_COUNT] = {e.uss, e.upp, zs[s], e.beta_s, e.beta_p, e.alpha, e.gss,
                                        e.gpp, e.gsp, e.gp2, e.hsp, e.dd1, e.dd2, e.rho[0],
                                        e.rho[1], e.rho[2], heat[s], eisol[s]};
  for (int k = 0; k < SGB_PARAM_COUNT; ++k) v[k] = vals[k];
  return SGB_OK;
}

size_t sgb_ctx_bytes_in_use(const sgb_ctx* ctx) { return ctx ? ctx->in_use : 0; }

int sgb_ctx_create(int device, size_t budget, sgb_ctx** out) {
  if (!out) return SGB_E_ARG;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || device < 0 || device >= n) return SGB_E_CUDA;
  auto* c = new sgb_ctx();
  c->device = device;
  c->budget = budget;
  if ((e = cudaSetDevice(device)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = upload_tables()) != cudaSuccess || (e = prepare_kernels()) != cudaSuccess ||
      (e = prepare_grid_purify()) != cudaSuccess ||
      (e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) {
    delete c;
    return SGB_E_CUDA;
  }
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  c->smem_optin = optin;
  if (cudaHostAlloc(&c->staging, kStagingBytes, cudaHostAllocDefault) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->staging_ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    sgb_ctx_destroy(c);
    return SGB_E_CUDA;
  }
  c->staging_bytes = kStagingBytes;
  for (int k = 0; k < 8; ++k) {
    cudaEvent_t ev;
    if (cudaEventCreate(&ev) != cudaSuccess) {
      sgb_ctx_destroy(c);
      return SGB_E_CUDA;
    }
    c->events.push_back(ev);
  }
  for (int k = 0; k < kNumClasses; ++k) {
    c->class_threads[k] = kClasses[k].threads;
    if (cudaStreamCreateWithFlags(&c->aux[k], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->joined[k], cudaEventDisableTiming) != cudaSuccess) {
      sgb_ctx_destroy(c);
      return SGB_E_CUDA;
    }
  }
  c->solver = default_solver();
  if (const char* env = getenv("SGB_CLASS_THREADS")) {  // e.g. "128,256,512,512,512"
    int k = 0;
    for (const char* p = env; *p && k < kNumClasses; ++k) {
      const int t = atoi(p);
      if (class_threads_ok(k, t)) c->class_threads[k] = t;
      while (*p && *p != ',') ++p;
      if (*p == ',') ++p;
    }
  }
  *out = c;
  return SGB_OK;
}

int sgb_ctx_set_density_solver(sgb_ctx* ctx, int solver) {
  if (!ctx) return SGB_E_ARG;
  if (solver != SGB_SOLVER_PURIFY && solver != SGB_SOLVER_JACOBI &&
      solver != SGB_SOLVER_PURIFY_MIXED)
    return fail(ctx, SGB_E_ARG, "unknown density solver %d", solver);
  ctx->solver = solver == SGB_SOLVER_JACOBI         ? SOLVER_JACOBI
                : solver == SGB_SOLVER_PURIFY_MIXED ? SOLVER_PURIFY_MIXED
                                                    : SOLVER_PURIFY;
  return SGB_OK;
}

int sgb_size_classes(int* count, int* nao_max, int* threads, int max_count) {
  if (!count) return SGB_E_ARG;
  *count = kNumClasses;
  for (int k = 0; k < kNumClasses && k < max_count; ++k) {
    if (nao_max) nao_max[k] = kClasses[k].nmax;
    if (threads) threads[k] = kClasses[k].threads;
  }
  return SGB_OK;
}

int sgb_ctx_set_class_threads(sgb_ctx* ctx, int count, const int* threads) {
  if (!ctx || !threads || count < 0 || count > kNumClasses) return SGB_E_ARG;
  for (int k = 0; k < count; ++k)
    if (!class_threads_ok(k, threads[k]))
      return fail(ctx, SGB_E_ARG, "size class %d cannot run %d-thread CTAs", k, threads[k]);
  for (int k = 0; k < count; ++k) ctx->class_threads[k] = threads[k];
  return SGB_OK;
}

int sgb_ctx_set_diis(sgb_ctx* ctx, int depth) {
  if (!ctx || depth < 0 || depth > 8 || depth == 1) return SGB_E_ARG;
  ctx->diis = depth;
  return SGB_OK;
}

int sgb_grid_configs(int* count, int* bm, int* warps, int* kblocks, int* stages, int max_count) {
  if (count) *count = kNumGridConfigs;
  for (int k = 0; k < kNumGridConfigs && k < max_count; ++k) {
    if (bm) bm[k] = kGridConfigs[k].bm;
    if (warps) warps[k] = kGridConfigs[k].warps;
    if (kblocks) kblocks[k] = kGridConfigs[k].kb;
    if (stages) stages[k] = kGridConfigs[k].stages;
  }
  return SGB_OK;
}

int sgb_ctx_set_grid_config(sgb_ctx* ctx, int config) {
  if (!ctx || config < -1 || config >= kNumGridConfigs) return SGB_E_ARG;
  ctx->grid_config = config;
  return SGB_OK;
}

int sgb_ctx_set_damping(sgb_ctx* ctx, double factor) {
  if (!ctx || !(factor >= 0.0 && factor < 1.0)) return SGB_E_ARG;
  ctx->damping = factor;
  return SGB_OK;
}

int sgb_ctx_set_limits(sgb_ctx* ctx, int max_sweeps, long long wait_spins) {
  if (!ctx || max_sweeps < 0) return SGB_E_ARG;
  ctx->max_sweeps = max_sweeps;
  ctx->wait_spins = wait_spins < 0 ? -1 : wait_spins;
  return SGB_OK;
}

int sgb_diag_barrier_timeout(sgb_ctx* ctx, int blocks, int extra, long long spins,
                             int* timed_out) {
  if (!ctx || blocks < 1 || extra < 0 || spins < 0 || !timed_out) return SGB_E_ARG;
  if (blocks > ctx->num_sms) return fail(ctx, SGB_E_ARG, "at most %d blocks", ctx->num_sms);
  char* mem = nullptr;
  size_t got = 0;
  if (int rc = arena_get(ctx, 256, "barrier probe", &mem, &got)) return rc;
  cudaStream_t st = ctx->stream;
  unsigned* bar = reinterpret_cast<unsigned*>(mem);
  int* err = reinterpret_cast<int*>(mem + 16);
  int h = 0;
  cudaError_t e = cudaMemsetAsync(mem, 0, 32, st);
  if (e == cudaSuccess) {
    // one 32-thread block per SM at most, so every block is resident; a cooperative launch
    // guarantees it
    GridBarrier b{bar, bar + 1, err, spins, (unsigned)(blocks + extra)};
    void* args[] = {&b};
    e = cudaLaunchCooperativeKernel((void*)k_barrier_probe, blocks, 32, args, 0, st);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  arena_put(ctx, mem, got);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "barrier probe");
  *timed_out = h != 0;
  return SGB_OK;
}

int sgb_ctx_set_sm_share(sgb_ctx* ctx, double share) {
  if (!ctx || !(share > 0.0) || share > 1.0) return SGB_E_ARG;
  ctx->sm_limit = share >= 1.0 ? 0 : std::max(1, (int)(share * ctx->num_sms));
  return SGB_OK;
}

int sgb_ctx_set_priority(sgb_ctx* ctx, int high) {
  if (!ctx) return SGB_E_ARG;
  int least = 0, greatest = 0;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  CUDA_TRY(ctx, cudaDeviceGetStreamPriorityRange(&least, &greatest));
  const int prio = high ? greatest : least;
  // every launch and copy of the context reads ctx->stream / ctx->aux[] when it is issued, so
  // the streams can be replaced once the work queued on them has finished
  cudaStream_t* all[1 + kNumClasses];
  all[0] = &ctx->stream;
  for (int k = 0; k < kNumClasses; ++k) all[1 + k] = &ctx->aux[k];
  for (cudaStream_t* sp : all) {
    cudaStream_t fresh = nullptr;
    CUDA_TRY(ctx, cudaStreamCreateWithPriority(&fresh, cudaStreamNonBlocking, prio));
    if (*sp) {
      cudaStreamSynchronize(*sp);
      cudaStreamDestroy(*sp);
    }
    *sp = fresh;
  }
  return SGB_OK;
}

int sgb_ctx_reserve(sgb_ctx* ctx, size_t bytes) {
  if (!ctx) return SGB_E_ARG;
  if (ctx->pool_busy) return fail(ctx, SGB_E_STATE, "the reserved arena is in use by a batch");
  if (ctx->pool) {
    cudaFree(ctx->pool);
    ctx->in_use -= ctx->pool_bytes;
    ctx->pool = nullptr;
    ctx->pool_bytes = 0;
  }
  if (!bytes) return SGB_OK;
  if (ctx->budget && ctx->in_use + bytes > ctx->budget)
    return fail(ctx, SGB_E_NOMEM, "reserve %zu bytes: budget %zu, in use %zu", bytes, ctx->budget,
                ctx->in_use);
  cudaError_t e = cudaMalloc(&ctx->pool, bytes);
  if (e != cudaSuccess) {
    ctx->pool = nullptr;
    return fail(ctx, SGB_E_NOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  }
  ctx->pool_bytes = bytes;
  ctx->in_use += bytes;
  return SGB_OK;
}

int sgb_ctx_destroy(sgb_ctx* ctx) {
  if (!ctx) return SGB_E_ARG;
  cudaSetDevice(ctx->device);
  free_batch(ctx->cached);
  ctx->cached = nullptr;
  // molecules and batches still alive: their device memory goes now, their host parts stay
  // for their own destroy calls, which then no longer reach this context
  for (sgb_mol* m : ctx->mols) {
    free_grid_work(ctx, m);
    m->ctx = nullptr;
  }
  ctx->mols.clear();
  for (sgb_batch* b : ctx->batches) {
    if (b->arena && !b->from_pool) arena_put(ctx, b->arena, b->bytes);
    if (b->diis) arena_put(ctx, b->diis, b->diis_bytes);
    give_event(ctx, b->ev0);
    give_event(ctx, b->ev1);
    b->arena = nullptr;
    b->diis = nullptr;
    b->ev0 = b->ev1 = nullptr;
    b->ctx = nullptr;
  }
  ctx->batches.clear();
  if (ctx->pool) cudaFree(ctx->pool);
  {
    std::lock_guard<std::mutex> lock(ctx->spare_mutex);
    release_spares(ctx, 0, 0);
  }
  for (int k = 0; k < kNumClasses; ++k) {
    if (ctx->aux[k]) cudaStreamDestroy(ctx->aux[k]);
    if (ctx->joined[k]) cudaEventDestroy(ctx->joined[k]);
  }
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);  // staged copies may still be running
  if (ctx->staging) cudaFreeHost(ctx->staging);
  if (ctx->staging_ev) cudaEventDestroy(ctx->staging_ev);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  for (cudaEvent_t ev : ctx->events) cudaEventDestroy(ev);
  delete ctx;
  return SGB_OK;
}

int sgb_ctx_synchronize(sgb_ctx* ctx) {
  if (!ctx) return SGB_E_ARG;
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return SGB_OK;
}

// ---- one molecule ---------------------------------------------------------------------------
int sgb_mol_create(sgb_ctx* ctx, int natoms, const int* Z, const double* xyz, sgb_mol** out) {
  if (!ctx || !out) return SGB_E_ARG;
  *out = nullptr;
  sgb_batch* b = nullptr;
  int rc = build_batch(ctx, 1, &natoms, Z, xyz, 101, &b);
  if (rc) return rc;
  auto* m = new sgb_mol();
  m->ctx = ctx;
  ctx->mols.push_back(m);
  m->b = b;
  *out = m;
  return SGB_OK;
}

int sgb_mol_destroy(sgb_mol* mol) {
  if (!mol) return SGB_E_ARG;
  if (mol->ctx) {
    auto& v = mol->ctx->mols;
    v.erase(std::remove(v.begin(), v.end(), mol), v.end());
  }
  free_grid_work(mol->ctx, mol);
  free_batch(mol->b);
  delete mol;
  return SGB_OK;
}

int sgb_mol_set_path(sgb_mol* mol, int path) {
  if (!mol || path < SGB_PATH_AUTO || path > SGB_PATH_GRID) return SGB_E_ARG;
  mol->path = path;
  return SGB_OK;
}

int sgb_mol_info(const sgb_mol* mol, int* natoms, int* nao, int* nocc, long long* nblocks) {
  if (!mol) return SGB_E_ARG;
  const MolDesc& d = mol->b->desc[0];
  if (natoms) *natoms = d.natoms;
  if (nao) *nao = d.nao;
  if (nocc) *nocc = d.nocc;
  if (nblocks) *nblocks = d.nblk;
  return SGB_OK;
}

int sgb_two_center(sgb_ctx* ctx, sgb_mol* mol) {
  if (!ctx || !mol) return SGB_E_ARG;
  if (use_grid(mol)) {
    const MolView v = mol_view(mol->b);
    k_grid_integrals<<<grid_blocks(ctx, tri(v.natoms)), kGridThreads, 0, ctx->stream>>>(v);
    CUDA_TRY(ctx, cudaGetLastError());
  } else {
    int rc = launch_stages(ctx, mol->b, STAGE_INTS, 0.0, 0, 0);
    if (rc) return rc;
  }
  mol->ints_done = true;
  mol->hcore_done = mol->scf_done = false;
  return sgb_ctx_synchronize(ctx);
}

int sgb_hcore(sgb_ctx* ctx, sgb_mol* mol) {
  if (!ctx || !mol) return SGB_E_ARG;
  if (!mol->ints_done) return fail(ctx, SGB_E_STATE, "Hcore needs the two-center integrals");
  if (use_grid(mol)) {
    const MolView v = mol_view(mol->b);
    k_grid_hcore<<<grid_blocks(ctx, (int64_t)v.natoms * 10 + tri(v.natoms)), kGridThreads, 0,
                   ctx->stream>>>(v);
    CUDA_TRY(ctx, cudaGetLastError());
  } else {
    int rc = launch_stages(ctx, mol->b, STAGE_HCORE, 0.0, 0, 0);
    if (rc) return rc;
  }
  mol->hcore_done = true;
  return sgb_ctx_synchronize(ctx);
}

int sgb_scf(sgb_ctx* ctx, sgb_mol* mol, double tol, int max_iter, sgb_scf_result* res,
            double* energies) {
  if (!ctx || !mol || max_iter < 0 || !(tol >= 0.0)) return SGB_E_ARG;
  if (!mol->hcore_done) return fail(ctx, SGB_E_STATE, "SCF needs Hcore");
  if (max_iter > mol->b->hist_stride - 1)
    return fail(ctx, SGB_E_ARG, "max_iter %d above %d", max_iter, mol->b->hist_stride - 1);
  if (use_grid(mol)) {
    const int st = scf_grid(ctx, mol, tol, max_iter, res, energies);
    if (st < 0) return st;
    mol->scf_done = true;
    return st;
  }
  int rc = launch_stages(ctx, mol->b, STAGE_SCF, tol, max_iter, 1);
  if (rc) return rc;
  sgb_batch* b = mol->b;
  double e_el = 0.0;
  int it = 0, cv = 0, st = 0;
  CUDA_TRY(ctx, cudaMemcpyAsync(&e_el, b->d_eel, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaMemcpyAsync(&it, b->d_niter, 4, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaMemcpyAsync(&cv, b->d_conv, 4, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaMemcpyAsync(&st, b->d_status, 4, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (energies)
    CUDA_TRY(ctx, cudaMemcpy(energies, b->d_hist, 8 * (size_t)(it + 1), cudaMemcpyDeviceToHost));
  if (res) {
    res->e_el = e_el;
    res->n_iter = it;
    res->converged = cv;
    res->status = st == MOL_OK ? SGB_OK : st == MOL_EIG_FAILED ? SGB_E_EIG : SGB_E_NAN;
  }
  mol->scf_done = true;
  return st == MOL_OK ? SGB_OK : st == MOL_EIG_FAILED ? SGB_E_EIG : SGB_E_NAN;
}

int sgb_core_core(sgb_ctx* ctx, sgb_mol* mol, double* e_cc) {
  if (!ctx || !mol || !e_cc) return SGB_E_ARG;
  if (!mol->ints_done) return fail(ctx, SGB_E_STATE, "core-core needs the two-center integrals");
  if (use_grid(mol)) {
    int rc = ensure_grid_work(ctx, mol);
    if (rc) return rc;
    const MolView v = mol_view(mol->b);
    const int nb = grid_blocks(ctx, tri(v.natoms));
    k_grid_core_core<<<nb, kGridThreads, 0, ctx->stream>>>(v, mol->gw.partial);
    k_reduce_sum<<<1, 256, 0, ctx->stream>>>(mol->gw.partial, nb, mol->gw.scalars + 1);
    CUDA_TRY(ctx, cudaGetLastError());
    CUDA_TRY(ctx, cudaMemcpyAsync(e_cc, mol->gw.scalars + 1, 8, cudaMemcpyDeviceToHost, ctx->stream));
    return sgb_ctx_synchronize(ctx);
  }
  int rc = launch_stages(ctx, mol->b, STAGE_CC, 0.0, 0, 0);
  if (rc) return rc;
  CUDA_TRY(ctx, cudaMemcpyAsync(e_cc, mol->b->d_ecc, 8, cudaMemcpyDeviceToHost, ctx->stream));
  return sgb_ctx_synchronize(ctx);
}

int sgb_fock(sgb_ctx* ctx, sgb_mol* mol, const double* P, double* F, double* e_el) {
  if (!ctx || !mol || !P) return SGB_E_ARG;
  if (!mol->hcore_done) return fail(ctx, SGB_E_STATE, "Fock needs Hcore");
  sgb_batch* b = mol->b;
  const size_t np = (size_t)tri(b->desc[0].nao);
  CUDA_TRY(ctx, cudaMemcpyAsync(b->d_P, P, 8 * np, cudaMemcpyHostToDevice, ctx->stream));
  const double* e_src = b->d_eel;
  if (use_grid(mol)) {
    int rc = ensure_grid_work(ctx, mol);
    if (!rc) rc = grid_fock(ctx, mol, false);
    if (rc) return rc;
    e_src = mol->gw.scalars;
  } else {
    int rc = launch_stages(ctx, b, STAGE_FOCK, 0.0, 0, 0);
    if (rc) return rc;
  }
  if (F) CUDA_TRY(ctx, cudaMemcpyAsync(F, b->d_F, 8 * np, cudaMemcpyDeviceToHost, ctx->stream));
  if (e_el) CUDA_TRY(ctx, cudaMemcpyAsync(e_el, e_src, 8, cudaMemcpyDeviceToHost, ctx->stream));
  return sgb_ctx_synchronize(ctx);
}

int sgb_electronic_energy(sgb_ctx* ctx, int nao, const double* H, const double* F,
                          const double* P, double* e_el) {
  if (!ctx || nao <= 0 || !H || !F || !P || !e_el) return SGB_E_ARG;
  const int64_t np = tri(nao);
  const int nb = grid_blocks(ctx, np);
  const size_t mat = align_up(8 * (size_t)np);
  char* mem = nullptr;
  size_t got = 0;
  if (int rc = arena_get(ctx, 3 * mat + 8 * (size_t)(nb + 1), "energy inputs", &mem, &got))
    return rc;
  double* dH = reinterpret_cast<double*>(mem);
  double* dF = reinterpret_cast<double*>(mem + mat);
  double* dP = reinterpret_cast<double*>(mem + 2 * mat);
  double* part = reinterpret_cast<double*>(mem + 3 * mat);
  cudaStream_t st = ctx->stream;
  cudaError_t e = cudaMemcpyAsync(dH, H, 8 * np, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dF, F, 8 * np, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dP, P, 8 * np, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    k_energy_partials<<<nb, kGridThreads, 0, st>>>(np, dH, dF, dP, part);
    k_reduce_sum<<<1, 256, 0, st>>>(part, nb, part + nb);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(e_el, part + nb, 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  arena_put(ctx, mem, got);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "electronic energy");
  return SGB_OK;
}

int sgb_get(sgb_ctx* ctx, const sgb_mol* mol, int which, double* host, size_t count) {
  if (!ctx || !mol || !host) return SGB_E_ARG;
  if ((which == SGB_EIGVAL || which == SGB_EIGVEC) && mol->eig_pending) {
    const int rc = grid_eigenpairs(ctx, const_cast<sgb_mol*>(mol));
    if (rc) return rc;
  }
  const sgb_batch* b = mol->b;
  const MolDesc& d = b->desc[0];
  const double* src = nullptr;
  size_t need = 0;
  switch (which) {
    case SGB_BLOCKS: src = b->d_ints; need = d.nblk; break;
    case SGB_HCORE: src = b->d_H; need = tri(d.nao); break;
    case SGB_FOCK: src = b->d_F; need = tri(d.nao); break;
    case SGB_DENSITY: src = b->d_P; need = tri(d.nao); break;
    case SGB_EIGVAL: src = b->d_eig; need = d.nao; break;
    case SGB_EIGVEC: src = b->d_T; need = (size_t)d.nao * d.nao; break;
    default: return fail(ctx, SGB_E_ARG, "unknown matrix id %d", which);
  }
  if (count < need) return fail(ctx, SGB_E_ARG, "buffer holds %zu, need %zu", count, need);
  CUDA_TRY(ctx, cudaMemcpyAsync(host, src, 8 * need, cudaMemcpyDeviceToHost, ctx->stream));
  return sgb_ctx_synchronize(ctx);
}

// ---- batches ---------------------------------------------------------------------------------
int sgb_batch_create(sgb_ctx* ctx, int nmol, const int* natoms, const int* Z, const double* xyz,
                     sgb_batch** out) {
  if (!ctx || !out) return SGB_E_ARG;
  *out = nullptr;
  return build_batch(ctx, nmol, natoms, Z, xyz, 0, out);
}

int sgb_batch_destroy(sgb_batch* b) {
  if (!b) return SGB_E_ARG;
  if (b->ctx && b->ctx->cached == b) b->ctx->cached = nullptr;
  free_batch(b);
  return SGB_OK;
}

int sgb_batch_set_coordinates(sgb_ctx* ctx, sgb_batch* b, const double* xyz) {
  if (!ctx || !b || !xyz) return SGB_E_ARG;
  const int64_t NA = b->natoms_total;
  const HostCopy up = {b->d_xyz, xyz, 24 * (size_t)NA};
  CUDA_TRY(ctx, upload(ctx, &up, 1, ctx->stream));
  k_ang_to_bohr<<<std::max<int64_t>(1, std::min<int64_t>((3 * NA + 255) / 256, 1024)), 256, 0,
                  ctx->stream>>>(b->d_xyz, b->d_pos, 3 * NA);
  CUDA_TRY(ctx, cudaGetLastError());
  return SGB_OK;
}

int sgb_batch_run(sgb_ctx* ctx, sgb_batch* b, double tol, int max_iter) {
  if (!ctx || !b || max_iter < 0 || !(tol >= 0.0)) return SGB_E_ARG;
  return launch_stages(ctx, b, STAGE_ALL, tol, max_iter, 0);
}

int sgb_batch_results(sgb_ctx* ctx, sgb_batch* b, double* e_el, double* e_cc, int* n_iter,
                      int* converged, int* status) {
  if (!ctx || !b) return SGB_E_ARG;
  const size_t n = (size_t)b->nmol;
  const HostCopy downs[] = {{e_el, b->d_eel, e_el ? 8 * n : 0},
                            {e_cc, b->d_ecc, e_cc ? 8 * n : 0},
                            {n_iter, b->d_niter, n_iter ? 4 * n : 0},
                            {converged, b->d_conv, converged ? 4 * n : 0},
                            {status, b->d_status, status ? 4 * n : 0}};
  CUDA_TRY(ctx, download(ctx, downs, 5, ctx->stream));
  CUDA_TRY(ctx, cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1));
  return SGB_OK;
}

int sgb_batch_last_ms(const sgb_batch* b, float* ms) {
  if (!b || !ms) return SGB_E_ARG;
  *ms = b->last_ms;
  return SGB_OK;
}

int sgb_batch_timestamps(sgb_ctx* ctx, sgb_batch* b, unsigned long long* t_begin,
                         unsigned long long* t_end) {
  if (!ctx || !b) return SGB_E_ARG;
  const size_t n = (size_t)b->nmol;
  const HostCopy downs[] = {{t_begin, b->d_tb, t_begin ? 8 * n : 0},
                            {t_end, b->d_te, t_end ? 8 * n : 0}};
  CUDA_TRY(ctx, download(ctx, downs, 2, ctx->stream));
  return SGB_OK;
}

int sgb_batch_launches(const sgb_batch* b, int* launches) {
  if (!b || !launches) return SGB_E_ARG;
  int n = 0;
  for (int c = 0; c < kNumClasses; ++c) n += b->class_count[c] > 0;
  *launches = n;
  return SGB_OK;
}

int sgb_batch_set_profiling(sgb_batch* b, int on) {
  if (!b) return SGB_E_ARG;
  b->profiling = on != 0;
  return SGB_OK;
}

int sgb_batch_stage_cycles(sgb_ctx* ctx, sgb_batch* b, unsigned long long* cycles) {
  if (!ctx || !b || !cycles) return SGB_E_ARG;
  if (!b->profiling) return fail(ctx, SGB_E_STATE, "stage timers are off (sgb_batch_set_profiling)");
  const HostCopy down = {cycles, b->d_stage, 8 * (size_t)kStageSlots * b->nmol};
  CUDA_TRY(ctx, download(ctx, &down, 1, ctx->stream));
  return SGB_OK;
}

int sgb_batch_device_coordinates(sgb_batch* b, void** dptr) {
  if (!b || !dptr) return SGB_E_ARG;
  *dptr = b->d_xyz;
  return SGB_OK;
}

int sgb_gradient(sgb_ctx* ctx, int natoms, const int* Z, const double* xyz, double tol, int max_iter,
                 double step, double* e_tot, double* grad) {
  if (!ctx || natoms <= 0 || !Z || !xyz || !grad || !(step > 0.0) || !(tol >= 0.0) || max_iter < 1)
    return SGB_E_ARG;
  // the molecule and its 6 natoms displaced copies (+/- step along each coordinate), one batch
  const int nmol = 1 + 6 * natoms;
  const int64_t per = 3 * (int64_t)natoms;
  std::vector<int> na(nmol, natoms), zz((size_t)nmol * natoms);
  std::vector<double> xx((size_t)nmol * per);
  for (int m = 0; m < nmol; ++m) {
    std::copy(Z, Z + natoms, zz.begin() + (size_t)m * natoms);
    std::copy(xyz, xyz + per, xx.begin() + (size_t)m * per);
    if (m > 0) {
      const int64_t c = (m - 1) / 2;  // coordinate 3 atom + axis
      xx[(size_t)m * per + c] += (m - 1) % 2 == 0 ? step : -step;
    }
  }
  sgb_batch* b = nullptr;
  int rc = build_batch(ctx, nmol, na.data(), zz.data(), xx.data(), 0, &b);
  if (rc) return rc;
  std::vector<double> eel(nmol), ecc(nmol);
  std::vector<int> st(nmol), cv(nmol);
  rc = sgb_batch_run(ctx, b, tol, max_iter);
  if (!rc) rc = sgb_batch_results(ctx, b, eel.data(), ecc.data(), nullptr, cv.data(), st.data());
  free_batch(b);
  if (rc) return rc;
  for (int m = 0; m < nmol; ++m) {
    if (st[m] != MOL_OK)
      return fail(ctx, st[m] == MOL_EIG_FAILED ? SGB_E_EIG : SGB_E_NAN,
                  "gradient: SCF of geometry %d stopped (status %d)", m, st[m]);
    if (!cv[m])
      return fail(ctx, SGB_E_NOCONV, "gradient: SCF of geometry %d did not converge in %d steps", m,
                  max_iter);
  }
  if (e_tot) *e_tot = eel[0] + ecc[0];
  for (int64_t c = 0; c < per; ++c) {
    const int p = 1 + 2 * (int)c, q = p + 1;
    grad[c] = ((eel[p] + ecc[p]) - (eel[q] + ecc[q])) / (2.0 * step);
  }
  return SGB_OK;
}

int sgb_run_molecules(sgb_ctx* ctx, int nmol, const int* natoms, const int* Z, const double* xyz,
                      double tol, int max_iter, double* e_el, double* e_cc, int* n_iter,
                      int* converged, int* status) {
  if (!ctx || nmol <= 0 || !natoms || !Z || !xyz) return SGB_E_ARG;
  sgb_batch* b = ctx->cached;
  bool same = b && b->nmol == nmol && std::equal(natoms, natoms + nmol, b->natoms.begin());
  if (same) same = std::equal(b->Z.begin(), b->Z.end(), Z);
  int rc;
  if (same) {
    rc = sgb_batch_set_coordinates(ctx, b, xyz);
  } else {
    free_batch(ctx->cached);
    ctx->cached = nullptr;
    rc = build_batch(ctx, nmol, natoms, Z, xyz, 0, &b);
    if (!rc) ctx->cached = b;
  }
  if (rc) return rc;
  rc = sgb_batch_run(ctx, b, tol, max_iter);
  if (rc) return rc;
  return sgb_batch_results(ctx, b, e_el, e_cc, n_iter, converged, status);
}

int sgb_scf_noalloc(int natoms, const int* Z, const double* xyz, double tol, int max_iter,
                    void* stream, double* e_el, double* e_cc, int* n_iter, int* converged,
                    int* status) {
  if (natoms <= 0 || !Z || !xyz || max_iter < 0 || !(tol >= 0.0)) return SGB_E_ARG;
  if (natoms > kNoAllocMaxAtoms) {
    fprintf(stderr, "sgb_scf_noalloc: %d atoms, the allocation-free path takes at most %d\n",
            natoms, kNoAllocMaxAtoms);
    return SGB_E_UNSUPPORTED;
  }
  // host-side layout on the stack (no heap, no device allocation)
  NoAllocHeader h;
  memset(&h, 0, sizeof h);
  int nao = 0, nel = 0, nheavy = 0;
  int64_t roff = 0;
  for (int a = 0; a < natoms; ++a) {
    const int s = slot_of(Z[a]);
    if (s < 0) return SGB_E_ELEMENT;
    const bool heavy = s != 0;
    h.slot[a] = (int8_t)s;
    h.first[a] = nao;
    h.hb[a] = nheavy;
    h.row_off[a] = roff;
    const int nh = nheavy + (heavy ? 1 : 0), nl = a + 1 - nh;
    roff += (int64_t)nh * (heavy ? 100 : 10) + (int64_t)nl * (heavy ? 10 : 1);
    nao += heavy ? 4 : 1;
    nel += s == 0 ? 1 : (Z[a] - 2);
    nheavy += heavy ? 1 : 0;
  }
  if (nao > kNoAllocMaxNao) {
    fprintf(stderr, "sgb_scf_noalloc: %d atomic orbitals, the allocation-free path takes at most %d\n",
            nao, kNoAllocMaxNao);
    return SGB_E_UNSUPPORTED;
  }
  memcpy(h.xyz, xyz, sizeof(double) * 3 * natoms);
  // device layout inside the static scratch
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off = align_up(off + bytes); return o; };
  const size_t o_head = take(sizeof(NoAllocHeader)), o_pos = take(24 * (size_t)natoms),
               o_res = take(sizeof(NoAllocResults)), o_ints = take(8 * (size_t)roff),
               o_H = take(8 * (size_t)tri(nao)), o_P = take(8 * (size_t)tri(nao)),
               o_F = take(8 * (size_t)tri(nao)), o_V = take(8 * (size_t)nao * nao),
               o_T = take(8 * (size_t)nao * nao), o_eig = take(8 * (size_t)nao);
  if (off > kNoAllocScratchBytes) {
    fprintf(stderr, "sgb_scf_noalloc: molecule needs %zu bytes of scratch, %zu available\n", off,
            kNoAllocScratchBytes);
    return SGB_E_UNSUPPORTED;
  }
  // per-device set-up on the first call: constant tables and the scratch's device address
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return SGB_E_CUDA;
  NoAllocDevice& nd = g_noalloc[dev];
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!nd.ready) {
      void* ptr = nullptr;
      if (upload_tables() != cudaSuccess || prepare_kernels() != cudaSuccess) return SGB_E_CUDA;
      if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return SGB_E_CUDA;
      if (cudaDeviceGetAttribute(&nd.num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return SGB_E_CUDA;
      nd.scratch = static_cast<unsigned char*>(ptr);
      nd.ready = true;
    }
  }
  unsigned char* base = nd.scratch;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  h.desc.natoms = natoms;
  h.desc.nao = nao;
  h.desc.nocc = nel / 2;
  h.desc.nheavy = nheavy;
  h.desc.nblk = roff;  // all offsets of the views below are relative to their own buffers
  h.desc.wmap = -1;
  h.order = 0;         // counter[] stays zero: it must start at zero every run
  if (cudaMemcpyAsync(base + o_head, &h, sizeof h, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return SGB_E_CUDA;
  NoAllocHeader* dh = reinterpret_cast<NoAllocHeader*>(base + o_head);
  double* pos = reinterpret_cast<double*>(base + o_pos);
  k_ang_to_bohr<<<1, 128, 0, st>>>(dh->xyz, pos, 3 * natoms);
  NoAllocResults* dr = reinterpret_cast<NoAllocResults*>(base + o_res);
  BatchArgs a;
  a.nmol = 1;
  a.mols = &dh->desc;
  a.order = &dh->order;
  a.counter = dh->counter;
  a.slot = dh->slot;
  a.pos = pos;
  a.first = dh->first;
  a.row_off = dh->row_off;
  a.hb = dh->hb;
  a.ints = reinterpret_cast<double*>(base + o_ints);
  a.H = reinterpret_cast<double*>(base + o_H);
  a.P = reinterpret_cast<double*>(base + o_P);
  a.F = reinterpret_cast<double*>(base + o_F);
  a.V = reinterpret_cast<double*>(base + o_V);
  a.T = reinterpret_cast<double*>(base + o_T);
  a.eig = reinterpret_cast<double*>(base + o_eig);
  a.W = nullptr;
  a.wmaps = nullptr;
  a.e_el = &dr->e_el;
  a.e_cc = &dr->e_cc;
  a.n_iter = &dr->n_iter;
  a.converged = &dr->converged;
  a.status = &dr->status;
  a.hist = nullptr;
  a.hist_stride = 0;
  a.tol = tol;
  a.max_iter = max_iter;
  a.nmax = nao;
  a.mat_doubles = mat_doubles_for(nao);
  a.sorted_vectors = 0;
  a.solver = default_solver();
  a.stages = STAGE_ALL;
  a.t_begin = nullptr;
  a.t_end = nullptr;
  a.stage_cycles = nullptr;
  const int c = class_of(nao);
  const size_t smem = (a.mat_doubles + extra_doubles(a.nmax)) * sizeof(double);
  if (launch_class(nd.num_sms, a, kClasses[c].cr, kClasses[c].threads, smem, st) != cudaSuccess)
    return SGB_E_CUDA;
  NoAllocResults r;
  if (cudaMemcpyAsync(&r, dr, sizeof r, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return SGB_E_CUDA;
  if (e_el) *e_el = r.e_el;
  if (e_cc) *e_cc = r.e_cc;
  if (n_iter) *n_iter = r.n_iter;
  if (converged) *converged = r.converged;
  const int st_code = r.status == MOL_OK ? SGB_OK : r.status == MOL_EIG_FAILED ? SGB_E_EIG : SGB_E_NAN;
  if (status) *status = st_code;
  return st_code;
}

}  // extern "C"
