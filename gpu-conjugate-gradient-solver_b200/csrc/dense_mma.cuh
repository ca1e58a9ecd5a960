// Coarsest-level solve x = A^-1 b with the packed lower triangle of A^-1 in
// FP16 tiles (one FP32 scale per tile), products on the tensor cores.
//
// The packed apply is a matrix-vector product: every tile element is used
// twice (A_IJ x_J for tile row I and, off the diagonal, A_IJ^T x_I for tile
// row J) and nothing else, so it is bound by the bytes of the tiles. With
// the products on the CUDA cores, a 64 x 64 FP16 tile costs more issue slots
// (conversions, 32 FMAs per thread, cross-lane reductions) than its 8 KB take
// to arrive. Here one warp handles one tile at a time with mma.sync
// m16n8k16 (FP16 in, FP32 accumulate): 16 MMAs for A_IJ x_J and 16 for
// A_IJ^T x_I, the operands read from shared memory by ldmatrix (ldmatrix.trans
// for the transposed product, same staged tile), the reduction over a tile's
// columns done inside the MMA. The N = 8 columns of the MMA's B operand carry
// the vector as two parts: column 0 its FP16 value after a power-of-two scale
// of the 64-entry chunk (largest magnitude in [2^14, 2^15)), column 1 the FP16
// rounding of what that part missed, so the vector enters with about 22
// significant bits and only the matrix is rounded to FP16 (relative 2^-11,
// the storage precision of the tile). The other six columns are zero: the
// tensor cores have three orders of magnitude more throughput than this
// product needs. A pre-pass (dense_vec_kernel) converts each 64-entry chunk
// of the vector into its fragments once per apply; the tile loop loads them
// (two 16-byte loads on lanes 0-7) one tile ahead.
//
// Tiles reach shared memory through the bulk-copy engine (cp.async.bulk, 8 KB
// each, completion on an mbarrier per stage), kMmaStages deep per warp, the
// first ones requested before the wait on the predecessor kernel (the inverse
// does not change during a solve). Each tile's two 64-entry contributions
// land in their own partial slots (FP32), summed per row in slot order by
// dense_reduce_kernel, so the result is the same on every run.
//
// Tile layout (dense_mma_offset): the 64 x 64 tile is 4 x 4 blocks of
// 16 x 16, block (ib, kb) at (4 ib + kb) * 256; a block is four 8 x 8
// matrices (rh, ch) at (2 rh + ch) * 64, each row-major: every ldmatrix phase
// (8 rows of 16 bytes) reads 128 contiguous bytes, free of bank conflicts.
#pragma once

#include <cuda_fp16.h>

#include "bulk.cuh"
#include "kernels.cuh"

namespace gsb {

constexpr int kMmaWarps = 4;      // warps per CTA
constexpr int kMmaStages = 3;     // tiles in flight per warp
constexpr int kMmaTileHalves = kDenseTile * kDenseTile;
constexpr unsigned kMmaTileBytes = kMmaTileHalves * 2;

// Shared memory of one CTA: per warp kMmaStages tiles, then the mbarriers.
__host__ __device__ constexpr size_t dense_mma_smem() {
  return static_cast<size_t>(kMmaWarps) * kMmaStages * kMmaTileBytes + 8 * kMmaWarps * kMmaStages;
}

__device__ __forceinline__ void ldsm_x4(unsigned addr, unsigned &r0, unsigned &r1, unsigned &r2, unsigned &r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}

__device__ __forceinline__ void ldsm_x4_trans(unsigned addr, unsigned &r0, unsigned &r1, unsigned &r2, unsigned &r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}

// d += a (16 x 16, row) * b (16 x 8, col), FP16 in, FP32 accumulate
__device__ __forceinline__ void mma_16816(float d[4], const unsigned a[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned pack_half2(__half lo, __half hi) {
  return static_cast<unsigned>(__half_as_ushort(lo)) | (static_cast<unsigned>(__half_as_ushort(hi)) << 16);
}

// B fragments of one 64-entry chunk of the vector (entries base .. base+63,
// zero past n): for k-block kb, lane (g, t) = (lane / 4, lane % 4) holds
// B[2t, 2t+1][g] and B[2t+8, 2t+9][g]; column 0 is the scaled FP16 part,
// column 1 its FP16 remainder, the rest zero. Returns the scale's inverse.
template <typename BT>
__device__ __forceinline__ float vector_fragments(const BT *__restrict__ b, int n, int base, int lane,
                                                  unsigned frag[4][2]) {
  const int g = lane >> 2, t = lane & 3;
  float v[4][4];
  float m = 0.f;
#pragma unroll
  for (int kb = 0; kb < 4; ++kb)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int i = base + kb * 16 + 2 * t + (e & 1) + (e >> 1) * 8;
      v[kb][e] = (g < 2 && i < n) ? float(b[i]) : 0.f;
      m = fmaxf(m, fabsf(v[kb][e]));
    }
  // lanes 0-3 (and 4-7) hold the whole chunk: the largest magnitude over them
  m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 1));
  m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 2));
  int ex = 0;
  if (m > 0.f) {
    frexpf(m, &ex);  // m = f 2^ex, f in [0.5, 1)
    ex = max(-100, min(100, ex));
  }
  const float s = ldexpf(1.f, 15 - ex), inv = ldexpf(1.f, ex - 15);
#pragma unroll
  for (int kb = 0; kb < 4; ++kb) {
    __half h[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const float y = v[kb][e] * s;
      const __half hi = __float2half_rn(y);
      h[e] = g == 0 ? hi : __float2half_rn(y - __half2float(hi));
    }
    frag[kb][0] = g < 2 ? pack_half2(h[0], h[1]) : 0u;
    frag[kb][1] = g < 2 ? pack_half2(h[2], h[3]) : 0u;
  }
  return __shfl_sync(0xffffffffu, inv, 0);  // lanes past 7 saw no entry
}

// One warp per 64-entry chunk c of the vector: its B fragments for lanes
// 0-7 (4 k-blocks x 2 registers, as two uint4 at frag[2 (8 c + lane)]) and
// the inverse of its scale (inv[c]). Converting each chunk once per apply
// keeps the conversion out of the tile loop, where every chunk is used by
// about `tiles` tiles.
template <typename BT>
__global__ void __launch_bounds__(256) dense_vec_kernel(int n, int tiles, const BT *__restrict__ b,
                                                        uint4 *__restrict__ frag, float *__restrict__ inv,
                                                        const int *done) {
  if (pass_entry(done)) return;
  const int lane = threadIdx.x & 31;
  const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (c >= tiles) return;
  unsigned f[4][2];
  const float iv = vector_fragments(b, n, c * kDenseTile, lane, f);
  if (lane < 8) {
    frag[2 * (8 * c + lane)] = make_uint4(f[0][0], f[0][1], f[1][0], f[1][1]);
    frag[2 * (8 * c + lane) + 1] = make_uint4(f[2][0], f[2][1], f[3][0], f[3][1]);
  }
  if (lane == 0) inv[c] = iv;
}

// The fragments of chunk c for this lane (zero past lane 7) and its inverse
// scale.
struct ChunkFrag {
  uint4 lo, hi;
  float inv;
};

__device__ __forceinline__ void load_chunk(const uint4 *__restrict__ frag, const float *__restrict__ inv, int c,
                                           int lane, ChunkFrag &f) {
  f.lo = f.hi = make_uint4(0u, 0u, 0u, 0u);
  if (lane < 8) {
    f.lo = __ldg(frag + 2 * (8 * c + lane));
    f.hi = __ldg(frag + 2 * (8 * c + lane) + 1);
  }
  f.inv = __ldg(inv + c);
}

__device__ __forceinline__ void chunk_b(const ChunkFrag &f, int kb, unsigned &b0, unsigned &b1) {
  const uint4 &u = kb < 2 ? f.lo : f.hi;
  b0 = (kb & 1) ? u.z : u.x;
  b1 = (kb & 1) ? u.w : u.y;
}

// Tile t of the packed lower triangle -> (I, J), I >= J (see dense_tile_of);
// next_tile steps to t + step along the rows.
__device__ __forceinline__ void next_tile(int &I, int &J, int step) {
  J += step;
  while (J > I) {
    J -= I + 1;
    ++I;
  }
}

// One warp per tile at a time: warp w of the grid takes tiles w, w + W, ...
// (W warps in the grid). Row contributions of tile (I, J) go to
// partial[(I * tiles + J) * 64 + r], column contributions (I != J) to
// partial[(J * tiles + I) * 64 + c].
static __global__ void __launch_bounds__(32 * kMmaWarps) dense_mma_kernel(int tiles, const __half *__restrict__ packed,
                                                                  const float *__restrict__ scales,
                                                                  const uint4 *__restrict__ frag,
                                                                  const float *__restrict__ inv,
                                                                  float *__restrict__ partial, CgState *st) {
  extern __shared__ __align__(128) unsigned char mma_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long total = static_cast<long long>(tiles) * (tiles + 1) / 2;
  const int W = gridDim.x * kMmaWarps;
  const long long first = static_cast<long long>(blockIdx.x) * kMmaWarps + warp;
  unsigned char *stage0 = mma_smem + static_cast<size_t>(warp) * kMmaStages * kMmaTileBytes;
  unsigned long long *bars =
      reinterpret_cast<unsigned long long *>(mma_smem + static_cast<size_t>(kMmaWarps) * kMmaStages * kMmaTileBytes) +
      warp * kMmaStages;
  // the first tiles are requested before the wait on the predecessor
  if (lane == 0) {
    for (int k = 0; k < kMmaStages; ++k) {
      mbar_init(&bars[k], 1);
      const long long t = first + static_cast<long long>(k) * W;
      if (t < total) {
        mbar_expect_tx(&bars[k], kMmaTileBytes);
        bulk_copy(stage0 + k * kMmaTileBytes, packed + t * kMmaTileHalves, kMmaTileBytes, &bars[k]);
      }
    }
  }
  __syncwarp();
  // a stopped solve, or a wait that gave up, still lets every requested copy
  // land before the warp leaves (bounded again)
  auto drain = [&](long long from) {
    if (lane == 0)
      for (long long i = from; i < from + kMmaStages; ++i)
        if (first + i * W < total) mbar_wait_bounded(&bars[i % kMmaStages], static_cast<unsigned>((i / kMmaStages) & 1));
  };
  if (pass_entry(&st->done)) {
    drain(0);
    return;
  }
  const int g = lane >> 2, t4 = lane & 3, q = lane >> 3, r8 = lane & 7;
  int I = 0, J = 0;
  ChunkFrag fj, fi;
  float sc = 0.f;
  if (first < total) {
    dense_tile_of(first, I, J);
    load_chunk(frag, inv, J, lane, fj);
    load_chunk(frag, inv, I, lane, fi);
    sc = __ldg(scales + first);
  }
  for (long long i = 0; first + i * W < total; ++i) {
    const long long t = first + i * W;
    const int k = static_cast<int>(i % kMmaStages);
    // the next tile's vector chunks and scale (from L2) are requested before
    // this tile's products
    int In = I, Jn = J;
    ChunkFrag fjn = fj, fin = fi;
    float scn = sc;
    const bool more = t + W < total;
    if (more) {
      next_tile(In, Jn, W);
      load_chunk(frag, inv, Jn, lane, fjn);
      load_chunk(frag, inv, In, lane, fin);
      scn = __ldg(scales + t + W);
    }
    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&bars[k], static_cast<unsigned>((i / kMmaStages) & 1)))) {
      if (lane == 0) {
        atomicExch(&st->sync_fault, 1);
        atomicExch(&st->done, 1);
      }
      drain(i);  // this tile's copy and the two after it
      return;
    }
    const unsigned tile = smem_addr(stage0 + k * kMmaTileBytes);
    // row product: rows of tile row I, k over the columns (x_J)
    float dr[4][4];
#pragma unroll
    for (int mb = 0; mb < 4; ++mb) {
      dr[mb][0] = dr[mb][1] = dr[mb][2] = dr[mb][3] = 0.f;
#pragma unroll
      for (int kb = 0; kb < 4; ++kb) {
        // matrices (rh, ch) = (q & 1, q >> 1): the A operand's register order
        const int m = (q & 1) * 2 + (q >> 1);
        unsigned a[4];
        ldsm_x4(tile + 2u * static_cast<unsigned>((mb * 4 + kb) * 256 + m * 64 + r8 * 8), a[0], a[1], a[2], a[3]);
        unsigned b0, b1;
        chunk_b(fj, kb, b0, b1);
        mma_16816(dr[mb], a, b0, b1);
      }
    }
    // transposed product: rows of tile row J (the tile's columns), k over
    // the tile's rows (x_I); block (ki, mj) transposed, matrices (q >> 1, q & 1)
    float dc[4][4];
    const bool off = I != J;
    if (off) {
#pragma unroll
      for (int mj = 0; mj < 4; ++mj) {
        dc[mj][0] = dc[mj][1] = dc[mj][2] = dc[mj][3] = 0.f;
#pragma unroll
        for (int ki = 0; ki < 4; ++ki) {
          unsigned a[4];
          ldsm_x4_trans(tile + 2u * static_cast<unsigned>((ki * 4 + mj) * 256 + q * 64 + r8 * 8), a[0], a[1], a[2],
                        a[3]);
          unsigned b0, b1;
          chunk_b(fi, ki, b0, b1);
          mma_16816(dc[mj], a, b0, b1);
        }
      }
    }
    // the stage is free once every lane's ldmatrix has returned: refill it
    __syncwarp();
    if (lane == 0 && t + static_cast<long long>(kMmaStages) * W < total) {
      fence_proxy_async_smem();
      mbar_expect_tx(&bars[k], kMmaTileBytes);
      bulk_copy(stage0 + k * kMmaTileBytes, packed + (t + static_cast<long long>(kMmaStages) * W) * kMmaTileHalves,
                kMmaTileBytes, &bars[k]);
    }
    // column 0 (scaled part) + column 1 (its remainder), rows g and g + 8
    if (t4 == 0) {
      float *pr = partial + (static_cast<size_t>(I) * tiles + J) * kDenseTile;
      const float fr = sc * fj.inv;
#pragma unroll
      for (int mb = 0; mb < 4; ++mb) {
        pr[mb * 16 + g] = (dr[mb][0] + dr[mb][1]) * fr;
        pr[mb * 16 + g + 8] = (dr[mb][2] + dr[mb][3]) * fr;
      }
      if (off) {
        float *pc = partial + (static_cast<size_t>(J) * tiles + I) * kDenseTile;
        const float fc = sc * fi.inv;
#pragma unroll
        for (int mj = 0; mj < 4; ++mj) {
          pc[mj * 16 + g] = (dc[mj][0] + dc[mj][1]) * fc;
          pc[mj * 16 + g + 8] = (dc[mj][2] + dc[mj][3]) * fc;
        }
      }
    }
    I = In, J = Jn, fj = fjn, fi = fin, sc = scn;
  }
}

}  // namespace gsb
