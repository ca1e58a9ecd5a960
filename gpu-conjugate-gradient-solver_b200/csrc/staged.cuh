// 3x3 block Gauss-Seidel colour pass with the slice's blocks staged in shared
// memory by the bulk-copy engine (BELL-32, one lane per node).
//
// The register form (bell_gs_kernel) streams a slice's block slots in groups
// of 8: a group costs a round trip for the block columns and values and then
// one for the neighbour gathers; a fine level of an elasticity problem (26
// off-diagonal blocks per node) needs four groups per slice, eight dependent
// round trips per warp, with 16 warps per SM (the values take ~128
// registers). Here one lane of the warp asks the bulk-copy engine
// (cp.async.bulk, global -> shared, completion counted on an mbarrier) for
// the whole slice at once: its block columns and its component-major block
// values, contiguous in the BELL layout. While they land, every lane fetches
// its node's right-hand side, own iterate and inverse diagonal block into
// registers; then the columns and values are read from shared memory
// (lane-contiguous, no bank conflict), only the neighbour gathers go to L2
// (16 slots per round trip: the values no longer occupy registers), and the
// row update is the register kernel's arithmetic in the same order (same
// iterate bits). A block holds two slices, so the blocks resident on an SM
// overlap one block's gathers with the others' copies.
//
// The mbarrier wait is bounded: after kBulkSpinLimit polls the warp gives
// up (the lanes vote, so the warp decides as one), sets CgState::sync_fault
// and stops the solve; before the warp leaves, its lane 0 waits (bounded
// again) for the copy in flight, so no bulk copy is left writing into the
// shared memory of a finished block.
#pragma once

#include "bulk.cuh"
#include "kernels.cuh"

namespace gsb {

constexpr int kStagedWarps = 2;                     // warps (slices) per block
constexpr int kStagedGroup = 16;                    // block slots gathered per round trip
// Shared memory of one warp: the mbarrier, then the columns and the values
// of a slice of `max_slots` (>= 1) block slots per lane (128-byte aligned
// parts).
template <typename T>
__host__ __device__ constexpr size_t staged_warp_bytes(int max_slots) {
  return 128 + ((static_cast<size_t>(max_slots) * 32 * 4 + 127) / 128) * 128 +
         static_cast<size_t>(max_slots) * 32 * 9 * sizeof(T);
}

template <typename T, typename BT, bool kZero, bool kRel = false>
__global__ void __launch_bounds__(32 * kStagedWarps) bell_gs_staged_kernel(
    BellView<T> A, int s_begin, int s_end, int node_begin, const BT *__restrict__ b, T *__restrict__ x,
    const T *__restrict__ wts, T omega, CgState *st, const T *__restrict__ nw, int max_slots,
    const T *__restrict__ xprev = nullptr, int node_end = 0) {
  extern __shared__ __align__(128) unsigned char staged_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int s = s_begin + blockIdx.x * kStagedWarps + warp;
  const bool active = s < s_end;  // uniform over the warp
  unsigned char *base = staged_smem + static_cast<size_t>(warp) * staged_warp_bytes<T>(max_slots);
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(base);
  int *scol = reinterpret_cast<int *>(base + 128);
  T *sval = reinterpret_cast<T *>(base + 128 + ((static_cast<size_t>(max_slots) * 32 * 4 + 127) / 128) * 128);
  int q0 = 0, q1 = 0, n0 = 0, n1 = 0;
  if (active) {
    q0 = __ldg(A.bptr + s), q1 = __ldg(A.bptr + s + 1), n0 = __ldg(A.srow + s), n1 = __ldg(A.srow + s + 1);
    if (lane == 0) {
      const unsigned cbytes = static_cast<unsigned>(q1 - q0) * 4u;
      const unsigned vbytes = static_cast<unsigned>(q1 - q0) * 9u * static_cast<unsigned>(sizeof(T));
      mbar_init(bar, 1);
      mbar_expect_tx(bar, cbytes + vbytes);
      if (cbytes > 0) {
        bulk_copy(scol, A.col + q0, cbytes, bar);
        bulk_copy(sval, A.val + 9 * static_cast<size_t>(q0), vbytes, bar);
      }
    }
  }
  __syncwarp();
  NodeBlocks<T> nb;
  if (active) fetch_node_blocks(A.dinv, n0, n1, lane, nb);
  // The copy and the inverse diagonal blocks (the matrix does not change
  // during a solve) are requested before the wait on the predecessor pass,
  // so under programmatic dependent launch they arrive while it drains. A
  // stopped solve still lets the copy land before the warp leaves.
  if (pass_entry(&st->done)) {
    if (active && lane == 0) mbar_wait_bounded(bar);
    return;
  }
  // the node's own operands arrive while the slice's blocks are copied
  const int node = n0 + lane;
  const bool valid = active && node < n1;
  T bi[3] = {T(0), T(0), T(0)}, xi[3] = {T(0), T(0), T(0)}, di[9];
  if (valid) {
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      bi[r] = T(b[3 * node + r]);
      if (!kZero) xi[r] = x[3 * node + r];
    }
  }
  bool ok = true;
  if (active) ok = __all_sync(0xffffffffu, mbar_wait_bounded(bar));
  if (!ok) {
    if (lane == 0) {
      atomicExch(&st->sync_fault, 1);
      atomicExch(&st->done, 1);
      mbar_wait_bounded(bar);  // let the copy in flight finish before the block can leave
    }
    return;
  }
  T acc[3] = {T(0), T(0), T(0)};
  if (active) {
    const int slots = (q1 - q0) / 32;
    constexpr int kGroup = kStagedGroup;
    for (int g0 = 0; g0 < slots; g0 += kGroup) {
      int bc[kGroup];
      bool use[kGroup];
      T xv[kGroup][3];
#pragma unroll
      for (int u = 0; u < kGroup; ++u) {
        const bool in = g0 + u < slots;
        bc[u] = in ? scol[(g0 + u) * 32 + lane] : -1;
        use[u] = in && (!kZero || bc[u] < node_begin);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          xv[u][c] = use[u] ? nb_load<kRel>(x, xprev, 3 * node_begin, 3 * node_end, 3 * bc[u] + c) : T(0);
      }
#pragma unroll
      for (int u = 0; u < kGroup; ++u)
        if (use[u]) {
          const T *v = sval + (static_cast<size_t>(g0 + u) * 9) * 32 + lane;
#pragma unroll
          for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[r] = fma(v[(3 * r + c) * 32], xv[u][c], acc[r]);
        }
    }
  }
  // the inverse diagonal blocks through shared memory (the value area is
  // free now; it holds at least 288 entries, max_slots >= 1)
  if (active) {
    stage_node_blocks(nb, lane, sval);
#pragma unroll
    for (int e = 0; e < 9; ++e) di[e] = sval[9 * lane + e];
  }
  if (valid) {
    const T w = nw != nullptr ? __ldg(nw + node) : (wts != nullptr ? wts[0] : omega);
    const T r0 = bi[0] - acc[0], r1 = bi[1] - acc[1], r2 = bi[2] - acc[2];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      T nv = di[3 * r] * r0;
      nv = fma(di[3 * r + 1], r1, nv);
      nv = fma(di[3 * r + 2], r2, nv);
      x[3 * node + r] = kZero ? w * nv : (T(1) - w) * xi[r] + w * nv;
    }
  }
}

}  // namespace gsb
