// Memory layout shared by host and device code.
//
// A batch holds any number of molecules.  Atom data lives in batch-wide structure-of-arrays
// buffers; each molecule owns contiguous ranges of the integral arena, of the packed-matrix
// arenas (lower triangles, n(n+1)/2 doubles, element (i,j), i>=j, at i(i+1)/2+j — the
// reference's layout, mymemory.cpp:369-371), of the square arenas (n*n doubles, row-major)
// and of the per-AO vectors.  Offsets are 64-bit so a single molecule may exceed 2^31
// elements (C2000H2002 needs 2.4e8 integral doubles).
//
// Integral storage per molecule follows the reference's ragged [A][B<=A] array
// (twocenterintegral.cpp:55-107) flattened in that order: X-X blocks 10x10 (bra pair on the
// higher-index atom A), H-X and X-H blocks 1x10 holding (s_H s_H | pair on X), H-H blocks
// 1x1.  Within row A the offset of block B is computable from the number of heavy atoms
// before B, so no per-pair table is stored.
#pragma once
#include <cstdint>

namespace sgb {

struct MolDesc {
  int natoms, nao, nocc, nheavy;
  int64_t atom0;  // first atom in the batch-wide atom arrays
  int64_t blk0;   // first double of the molecule's integral blocks
  int64_t pk0;    // first double of its packed matrices
  int64_t sq0;    // first double of its square matrices
  int64_t ao0;    // first entry of its per-AO vectors
  int64_t nblk;   // integral doubles owned
  int64_t w0;     // first double of its work matrices in global memory (nao > 160)
  int wmap;       // its pair of work-matrix tensor maps (nao > 160), or -1
  int pad_;
};

// Block offset (relative to the molecule's blk0) of atom pair (A, B), A >= B.
__host__ __device__ inline int64_t block_offset(const int64_t* row_off, const int* heavy_before,
                                                const int8_t* slot, int A, int B) {
  const bool hA = slot[A] != 0;
  const int hb = heavy_before[B];
  return row_off[A] + (int64_t)hb * (hA ? 100 : 10) + (int64_t)(B - hb) * (hA ? 10 : 1);
}

__host__ __device__ inline int64_t row_size(const int* heavy_before, const int8_t* slot, int A) {
  const bool hA = slot[A] != 0;
  const int nh = heavy_before[A] + (hA ? 1 : 0);  // heavy atoms with index <= A
  const int nl = A + 1 - nh;
  return (int64_t)nh * (hA ? 100 : 10) + (int64_t)nl * (hA ? 10 : 1);
}

__host__ __device__ inline int64_t tri(int64_t i) { return i * (i + 1) / 2; }

// Packed lower-triangle index of (i, j) in either order.
__host__ __device__ inline int64_t pk(int i, int j) {
  return i >= j ? tri(i) + j : tri(j) + i;
}

// Z -> element slot (0 H, 1 C, 2 N, 3 O), -1 if MNDO has no parameters for it here.
__host__ __device__ inline int slot_of(int z) {
  return z == 1 ? 0 : z == 6 ? 1 : z == 7 ? 2 : z == 8 ? 3 : -1;
}

}  // namespace sgb
