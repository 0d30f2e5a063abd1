// kernels.cu -- sm_100a kernels of the BEADS per-step hot path.
//
// Reference behaviour followed (paths inside the reference project):
//   cell id             native/src/simulation/neighbor/cell_list_build.cu:110-166
//   neighbour inclusion native/src/simulation/neighbor/full/full_neighbor_path_common.cuh:49-94
//   stencils            full/regular_cell_neighbor_builder.cu:40-113,
//                       full/small_dimension_neighbor_builder.cu:56-142
//   rebuild policy      native/src/simulation/neighbor/neighbor_system.cpp:79-216
//   displacement check  native/src/simulation/neighbor/rebuild_tracker.cu:50-94
//   LJ pair             native/src/forcefield/pair/pair_lj.cu:21-192
//   harmonic bond       native/src/forcefield/bond/bond_harmonic.cu:24-99
//   harmonic angle      native/src/forcefield/angle/angle_harmonic.cu:23-178
//   harmonic dihedral   native/src/forcefield/dihedral/dihedral_harmonic.cu:22-227
//   velocity Verlet     native/src/dynamics/integrator/velocity_verlet.cu:59-111
//   Berendsen           native/src/dynamics/thermostat/berendsen_thermostat.cu:104-163
//
// Design (not a translation): every kernel runs over all replicas of a batch
// at once; a block never straddles two replicas; the rebuild decision is taken
// on the device so a captured step loop needs no host round trip; totals are
// reduced in 64-bit fixed point so they do not depend on block scheduling;
// bonded forces are gathered per particle (each thread evaluates the terms its
// particle belongs to) so no force atomics exist anywhere.
#include "kernels.cuh"
#include "device_util.cuh"

#include <cstdio>
#include <stdexcept>
#include <string>

namespace bb {
namespace {

// ---------------------------------------------------------------------------
// pre: Berendsen lambda of the previous step, half-kick, drift, wrap, image
// update, displacement check; k_decide then takes the rebuild decision for
// this step (neighbor_system.cpp:79-105).
template <int kMode>
__global__ void __launch_bounds__(kBlock)
k_pre(DeviceView v, float sd_dmax, float sd_fref) {
  wait_prior_grid();
  const uint32_t b = blockIdx.x;
  const uint32_t r = v.block_replica[b];
  const ReplicaParams& p = v.rp[r];
  ReplicaState* st = &v.rs[r];
  const uint32_t slot = b * kBlock + threadIdx.x;
  const uint32_t local = slot - p.atom_begin;
  const unsigned long long phys = st->step + 1ull;
  const bool check_step = (kMode == kPreDescent) || p.skin == 0.0f ||
                          (phys % (unsigned long long)p.check_every) == 0ull;
  const float lam = (kMode == kPreVerlet) ? (float)st->lambda : 1.0f;

  if (local < p.n_atoms) {
    float4 x = v.pos[slot];
    float4 vm = v.vel[slot];
    const float4 f = v.force[slot];
    if (kMode == kPreVerlet) {
      if (lam != 1.0f) {
        vm.x = __fmul_rn(vm.x, lam);
        vm.y = __fmul_rn(vm.y, lam);
        vm.z = __fmul_rn(vm.z, lam);
      }
      const float h = __fdiv_rn(__fmul_rn(0.5f, p.dt), vm.w);
      vm.x = __fmaf_rn(h, f.x, vm.x);
      vm.y = __fmaf_rn(h, f.y, vm.y);
      vm.z = __fmaf_rn(h, f.z, vm.z);
      x.x = __fmaf_rn(p.dt, vm.x, x.x);
      x.y = __fmaf_rn(p.dt, vm.y, x.y);
      x.z = __fmaf_rn(p.dt, vm.z, x.z);
      v.vel[slot] = vm;
    } else {
      const float fn = sqrtf(norm2(f.x, f.y, f.z));
      const float s = sd_dmax / fmaxf(fn, sd_fref);
      if (isfinite(s) && isfinite(fn)) {
        x.x = __fmaf_rn(s, f.x, x.x);
        x.y = __fmaf_rn(s, f.y, x.y);
        x.z = __fmaf_rn(s, f.z, x.z);
      }
    }
    const float cx = floorf(__fmul_rn(__fsub_rn(x.x, p.lo[0]), p.inv_len[0]));
    const float cy = floorf(__fmul_rn(__fsub_rn(x.y, p.lo[1]), p.inv_len[1]));
    const float cz = floorf(__fmul_rn(__fsub_rn(x.z, p.lo[2]), p.inv_len[2]));
    x.x = __fmaf_rn(-cx, p.len[0], x.x);
    x.y = __fmaf_rn(-cy, p.len[1], x.y);
    x.z = __fmaf_rn(-cz, p.len[2], x.z);
    v.pos[slot] = x;
    // Images and the crossing count change only on a boundary crossing, so
    // a step reads neither image vector otherwise.
    uint32_t cross = 0u;
    const bool crossed = cx != 0.0f || cy != 0.0f || cz != 0.0f;
    if (crossed) {
      int4 im = v.img[slot];
      im.x += (int)cx;
      im.y += (int)cy;
      im.z += (int)cz;
      v.img[slot] = im;
      const uint32_t c0 = v.cross[slot];
      cross = pack_cross(cross_field(c0, 0) + (int)cx, cross_field(c0, 1) + (int)cy,
                         cross_field(c0, 2) + (int)cz) | (c0 & kCrossSaturated);
      v.cross[slot] = cross;
    }
    if (check_step) {
      const float4 rx = v.ref_pos[slot];
      if (!crossed) cross = v.cross[slot];
      // (img - ref_img) L + (x - x_ref), the reference's displacement.
      const float dx = __fmaf_rn((float)cross_field(cross, 0), p.len[0], __fsub_rn(x.x, rx.x));
      const float dy = __fmaf_rn((float)cross_field(cross, 1), p.len[1], __fsub_rn(x.y, rx.y));
      const float dz = __fmaf_rn((float)cross_field(cross, 2), p.len[2], __fsub_rn(x.z, rx.z));
      if (norm2(dx, dy, dz) > p.disp_thr_sq || (cross & kCrossSaturated) != 0u) {
        st->exceeded = 1u;  // every writer stores the same value
      }
    }
  }
}

// pre, second part: one thread per replica takes the rebuild decision of
// this step from the displacement flag k_pre's blocks set (a separate launch
// instead of a last-block handshake: no fence and no same-address atomic in
// each of k_pre's blocks).
template <int kMode>
__global__ void k_decide(DeviceView v, cudaGraphConditionalHandle cond, int use_cond) {
  wait_prior_grid();
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= v.n_replicas) return;
  const ReplicaParams& p = v.rp[r];
  ReplicaState* st = &v.rs[r];
  const unsigned long long phys = st->step + 1ull;
  const bool check_step = (kMode == kPreDescent) || p.skin == 0.0f ||
                          (phys % (unsigned long long)p.check_every) == 0ull;
  const unsigned exceeded = st->exceeded;
  st->exceeded = 0u;
  unsigned need = 0u;
  if (st->status & (kStatusNonFinite | kStatusFixedOverflow)) {
    // The state has failed (non-finite velocities, or a value beyond the
    // fixed-point range): no more list builds for this replica, whose
    // coordinates may no longer be finite; the host raises at the end of the
    // chunk.
    need = 0u;
  } else if (kMode == kPreDescent || p.skin == 0.0f) {
    need = (kMode == kPreDescent) ? exceeded : 1u;
  } else if (check_step) {
    const bool first = st->checks_since_build == 0u;
    st->checks_since_build += 1u;
    if (exceeded) {
      need = 1u;
      if (p.check_every > 1u && first) st->dangerous += 1ull;
    }
  }
  if (need) {
    st->builds += 1ull;
    st->reorder_now = (p.sort_every > 0u && (st->builds % p.sort_every) == 0ull) ? 1u : 0u;
    st->checks_since_build = 0u;
  } else {
    st->reorder_now = 0u;
  }
  st->need_rebuild = need;
  // Inside a captured step the rebuild chain is the body of a conditional
  // graph node: any replica that rebuilds switches it on for this step.
  if (need && use_cond) cudaGraphSetConditional(cond, 1u);
  if (kMode == kPreVerlet) st->lambda = 1.0;
}

// Marks every replica for a rebuild (initial build / explicit eval).
__global__ void k_force_rebuild_flags(DeviceView v, int count_build) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= v.n_replicas) return;
  ReplicaState* st = &v.rs[r];
  const ReplicaParams& p = v.rp[r];
  st->need_rebuild = 1u;
  if (count_build) {
    st->builds += 1ull;
    st->reorder_now =
        (p.sort_every > 0u && (st->builds % p.sort_every) == 0ull) ? 1u : 0u;
  } else {
    st->reorder_now = 0u;
  }
  st->checks_since_build = 0u;
}

// rebuild 2: exclusive scan of the cell counts (the cell starts), in three
// kernels so that a replica with many cells is scanned by many blocks:
// k_scan_sum (one block per chunk of kScanChunk cells: the chunk's total),
// k_scan (one block per replica: the work list of the per-cell kernels and
// the exclusive prefix of the replica's chunk totals) and k_scan_cells (one
// block per chunk: the starts and cursors of its cells; the counts are reset
// for the next build).  When every replica fits one chunk, k_scan_single
// does all three in one launch.
constexpr int kScanThreads = 1024;
constexpr int kScanWarps = kScanThreads / 32;
constexpr uint32_t kScanPer = kScanChunk / kScanThreads;  // consecutive cells per thread

// Exclusive prefix of x over the block (kScanThreads threads) and the total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t& total) {
  __shared__ uint32_t ws[kScanWarps + 1];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t inc = x;
#pragma unroll
  for (uint32_t o = 1; o < 32u; o <<= 1) {
    const uint32_t up = __shfl_up_sync(kFull, inc, o);
    if (lane >= o) inc += up;
  }
  if (lane == 31u) ws[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const uint32_t t = ws[lane];
    uint32_t wi = t;
#pragma unroll
    for (uint32_t o = 1; o < 32u; o <<= 1) {
      const uint32_t up = __shfl_up_sync(kFull, wi, o);
      if (lane >= o) wi += up;
    }
    ws[lane] = wi - t;                     // warps before this one
    if (lane == 31u) ws[kScanWarps] = wi;  // the block total
  }
  __syncthreads();
  const uint32_t out = ws[warp] + inc - x;
  total = ws[kScanWarps];
  __syncthreads();  // ws is reused by the next call
  return out;
}

// ---------------------------------------------------------------------------
// The per-slot kernels of the rebuild chain (bin, scatter, reorder) touch
// only the replicas that rebuild.  In a batch, where a step typically
// rebuilds a fifth of the replicas, they walk a list of those replicas'
// 128-slot blocks with a grid of about one wave, instead of launching one
// block per slot block of the batch that mostly returns at once.  Block item
// w is block w - chain_block_start[q] of the rebuilding replica q with
// chain_block_start[q] <= w < chain_block_start[q + 1]; k_chain_blocks (one
// block) lays the list out at the head of the chain.
__global__ void __launch_bounds__(kScanThreads) k_chain_blocks(DeviceView v) {
  uint32_t run = 0;
  for (uint32_t base = 0; base < v.n_replicas; base += kScanThreads) {
    const uint32_t q = base + threadIdx.x;
    const uint32_t x = (q < v.n_replicas && v.rs[q].need_rebuild) ? v.rp[q].n_pad / kBlock : 0u;
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(x, total);
    if (q < v.n_replicas) v.chain_block_start[q] = run + ex;
    run += total;
  }
  if (threadIdx.x == 0) v.chain_block_start[v.n_replicas] = run;
}

// Runs F(v, b) for every slot block b this launch covers: the listed blocks
// of the rebuilding replicas (grid-stride over the list) or, without the
// list, block blockIdx.x of the batch.  F returns early for blocks of
// replicas that do not rebuild; it holds no barrier.
template <void (*F)(const DeviceView&, uint32_t)>
__device__ __forceinline__ void for_chain_blocks(const DeviceView& v) {
  if (v.chain_block_list) {
    const uint32_t* start = v.chain_block_start;
    const uint32_t total = start[v.n_replicas];
    for (uint32_t w = blockIdx.x; w < total; w += gridDim.x) {
      uint32_t lo = 0, hi = v.n_replicas;  // start[lo] <= w < start[hi]
      while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (start[mid] <= w) lo = mid; else hi = mid;
      }
      F(v, v.rp[lo].block_begin + (w - start[lo]));
    }
  } else {
    F(v, blockIdx.x);
  }
}

// rebuild 1: cell id and per-cell count.
__device__ __forceinline__ void bin_block(const DeviceView& v, uint32_t b) {
  const uint32_t r = v.block_replica[b];
  if (!v.rs[r].need_rebuild) return;
  const ReplicaParams& p = v.rp[r];
  const uint32_t slot = b * kBlock + threadIdx.x;
  const uint32_t local = slot - p.atom_begin;
  if (local >= p.n_atoms) return;
  const float4 x = v.pos[slot];
  const uint32_t ix = axis_cell(x.x, p.lo[0], p.inv_cell[0], p.nc[0]);
  const uint32_t iy = axis_cell(x.y, p.lo[1], p.inv_cell[1], p.nc[1]);
  const uint32_t iz = axis_cell(x.z, p.lo[2], p.inv_cell[2], p.nc[2]);
  const uint32_t cell = p.cell_begin + ix + p.nc[0] * (iy + p.nc[1] * iz);
  v.cell_of_slot[slot] = cell;
  atomicAdd(&v.cell_count[cell], 1u);
}

__global__ void __launch_bounds__(kBlock) k_bin(DeviceView v) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *v.chain_launches += 1ull;  // launches of the chain
  for_chain_blocks<bin_block>(v);
}

__global__ void __launch_bounds__(kScanThreads) k_scan_sum(DeviceView v) {
  const uint32_t b = blockIdx.x;
  const uint32_t r = v.scan_chunk_replica[b];
  if (!v.rs[r].need_rebuild) return;
  const ReplicaParams& p = v.rp[r];
  const uint32_t c0 = (b - v.scan_chunk_first[r]) * kScanChunk;
  const uint32_t* count = v.cell_count + p.cell_begin;
  uint32_t s = 0;
#pragma unroll
  for (uint32_t k = 0; k < kScanPer; ++k) {
    const uint32_t c = c0 + k * kScanThreads + threadIdx.x;
    if (c < p.n_cells) s += count[c];
  }
  s = __reduce_add_sync(kFull, s);
  __shared__ uint32_t part[kScanWarps];
  if ((threadIdx.x & 31u) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kScanWarps; ++w) t += part[w];
    v.scan_chunk_sum[b] = t;
  }
}

// Work list of the per-cell kernels (cell sort, list build): work item w is
// cell w - work_start[q] of the rebuilding replica q with work_start[q] <= w
// < work_start[q + 1].  Block r (one per replica) writes entry r (the cells
// of the rebuilding replicas before it), block 0 also the total.
__device__ __forceinline__ void write_work_start(const DeviceView& v, uint32_t r) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  {
    uint32_t before = 0, all = 0;
    for (uint32_t q = threadIdx.x; q < v.n_replicas; q += kScanThreads) {
      const uint32_t c = v.rs[q].need_rebuild ? v.rp[q].n_cells : 0u;
      all += c;
      before += q < r ? c : 0u;
    }
    before = __reduce_add_sync(kFull, before);
    all = __reduce_add_sync(kFull, all);
    __shared__ uint32_t part[2][kScanWarps];
    if (lane == 0) {
      part[0][warp] = before;
      part[1][warp] = all;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t sb = 0, sa = 0;
      for (int w = 0; w < kScanWarps; ++w) {
        sb += part[0][w];
        sa += part[1][w];
      }
      v.work_start[r] = sb;
      if (r == 0) v.work_start[v.n_replicas] = sa;
    }
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan(DeviceView v) {
  const uint32_t r = blockIdx.x;
  write_work_start(v, r);
  if (!v.rs[r].need_rebuild) return;  // block-uniform
  const ReplicaParams& p = v.rp[r];
  // Exclusive prefix of the replica's chunk totals, in place.
  const uint32_t f0 = v.scan_chunk_first[r], f1 = v.scan_chunk_first[r + 1];
  uint32_t run = 0;
  for (uint32_t base = f0; base < f1; base += kScanThreads) {
    const uint32_t at = base + threadIdx.x;
    const uint32_t x = at < f1 ? v.scan_chunk_sum[at] : 0u;
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(x, total);
    if (at < f1) v.scan_chunk_sum[at] = run + ex;
    run += total;
  }
  if (threadIdx.x == 0) v.cell_start[p.start_base + p.n_cells] = p.atom_begin + p.n_atoms;
}

// Starts and cursors of the cells of chunk `chunk` of replica p (the counts
// are reset for the next build); `prefix` is the count total of the
// replica's chunks before it.
__device__ __forceinline__ void scan_chunk_cells(const DeviceView& v, const ReplicaParams& p,
                                                 uint32_t chunk, uint32_t prefix) {
  const uint32_t c0 = chunk * kScanChunk + threadIdx.x * kScanPer;
  uint32_t* count = v.cell_count + p.cell_begin;
  uint32_t cnt[kScanPer];
  uint32_t s = 0;
#pragma unroll
  for (uint32_t k = 0; k < kScanPer; ++k) {
    cnt[k] = c0 + k < p.n_cells ? count[c0 + k] : 0u;
    s += cnt[k];
  }
  uint32_t total;
  uint32_t run = p.atom_begin + prefix + block_exclusive_scan(s, total);
  uint32_t* start = v.cell_start + p.start_base;
  uint32_t* cursor = v.cell_cursor + p.cell_begin;
#pragma unroll
  for (uint32_t k = 0; k < kScanPer; ++k) {
    const uint32_t c = c0 + k;
    if (c < p.n_cells) {
      start[c] = run;
      cursor[c] = run;
      count[c] = 0u;
    }
    run += cnt[k];
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_cells(DeviceView v) {
  const uint32_t b = blockIdx.x;
  const uint32_t r = v.scan_chunk_replica[b];
  if (!v.rs[r].need_rebuild) return;
  scan_chunk_cells(v, v.rp[r], b - v.scan_chunk_first[r], v.scan_chunk_sum[b]);
}

// The same scan when every replica's cells fit one chunk (a batch of small
// replicas): the work list, then the replica's starts and cursors with a
// zero chunk prefix, in one launch instead of three.
__global__ void __launch_bounds__(kScanThreads) k_scan_single(DeviceView v) {
  const uint32_t r = blockIdx.x;
  write_work_start(v, r);
  if (!v.rs[r].need_rebuild) return;  // block-uniform
  const ReplicaParams& p = v.rp[r];
  scan_chunk_cells(v, p, 0u, 0u);
  if (threadIdx.x == 0) v.cell_start[p.start_base + p.n_cells] = p.atom_begin + p.n_atoms;
}

// rebuild 3: scatter slots into their cells (order inside a cell is fixed by
// the next kernel).
__device__ __forceinline__ void scatter_block(const DeviceView& v, uint32_t b) {
  const uint32_t r = v.block_replica[b];
  if (!v.rs[r].need_rebuild) return;
  const ReplicaParams& p = v.rp[r];
  const uint32_t slot = b * kBlock + threadIdx.x;
  if (slot - p.atom_begin >= p.n_atoms) return;
  const uint32_t at = atomicAdd(&v.cell_cursor[v.cell_of_slot[slot]], 1u);
  v.cell_atoms[at] = slot;
}

__global__ void __launch_bounds__(kBlock) k_scatter(DeviceView v) {
  for_chain_blocks<scatter_block>(v);
}

// The replica of work item w (see k_scan); w is warp-uniform.
__device__ __forceinline__ uint32_t work_replica(const DeviceView& v, uint32_t w) {
  uint32_t lo = 0, hi = v.n_replicas;  // work_start[lo] <= w < work_start[hi]
  while (hi - lo > 1u) {
    const uint32_t mid = (lo + hi) >> 1;
    if (v.work_start[mid] <= w) {
      lo = mid;
    } else {
      hi = mid;
    }
  }
  return lo;
}

// rebuild 4: sort each cell's slots ascending, which makes the counting sort
// stable and the whole build deterministic.  One warp per cell; a bitonic
// network in registers for <= 32 members, a rank sort in shared memory up to
// 256, insertion sort beyond.  Also
// gathers the positions in cell order (pos2[q] = pos[cell_atoms[q]]), so the
// list build reads its candidates with contiguous loads that do not wait on
// the slot index; the reorder kernels find them there too.
constexpr uint32_t kSortRankMax = 256;  // cells up to this size: rank sort in shared memory
constexpr uint32_t kSortThreadMax = 8;  // sparse replicas: cells up to this size, one thread each
// Sorts cell c of replica p (one warp; keys: this warp's shared scratch).
__device__ __forceinline__ void sort_cell(const DeviceView& v, const ReplicaParams& p,
                                          uint32_t c, uint32_t lane, uint32_t* keys) {
  {
    const uint32_t s0 = v.cell_start[p.start_base + c];
    const uint32_t s1 = v.cell_start[p.start_base + c + 1];
    const uint32_t n = s1 - s0;
    if (p.sparse && n <= kSortThreadMax) return;  // sorted by k_cellsort_sparse
    if (n <= 32u) {
      uint32_t val = lane < n ? v.cell_atoms[s0 + lane] : 0xffffffffu;
      if (n > 1u) {
        for (uint32_t k = 2; k <= 32; k <<= 1) {
          for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            const uint32_t other = __shfl_xor_sync(kFull, val, j);
            const bool up = (lane & k) == 0u;
            const bool lower = (lane & j) == 0u;
            val = (lower == up) ? min(val, other) : max(val, other);
          }
        }
      }
      if (lane < n) {
        v.cell_atoms[s0 + lane] = val;
        v.pos2[s0 + lane] = v.pos[val];
      }
    } else if (n <= kSortRankMax) {
      // Rank sort in shared memory: the slots are distinct, so a slot's
      // place is the number of smaller slots in the cell.
      for (uint32_t q = lane; q < n; q += 32u) keys[q] = v.cell_atoms[s0 + q];
      __syncwarp();
      for (uint32_t q = lane; q < n; q += 32u) {
        const uint32_t key = keys[q];
        uint32_t rank = 0;
        for (uint32_t t = 0; t < n; ++t) rank += keys[t] < key ? 1u : 0u;
        v.cell_atoms[s0 + rank] = key;
        v.pos2[s0 + rank] = v.pos[key];
      }
    } else {
      // A crowded cell: its members in ascending slot order are the slots of
      // the replica whose cell is c, in the order a scan of the replica meets
      // them; the warp scans cell_of_slot 32 slots at a time and compacts the
      // matches by ballot (work linear in the replica's size, whatever the
      // occupancy).
      const uint32_t cg = p.cell_begin + c;
      const uint32_t lt = (1u << lane) - 1u;
      uint32_t at = s0;
      for (uint32_t b0 = p.atom_begin; b0 < p.atom_begin + p.n_atoms && at < s1; b0 += 32u) {
        const uint32_t s = b0 + lane;
        const bool in = s < p.atom_begin + p.n_atoms && v.cell_of_slot[s] == cg;
        const uint32_t m = __ballot_sync(kFull, in);
        if (in && at + __popc(m & lt) < s1) v.cell_atoms[at + __popc(m & lt)] = s;
        at += __popc(m);
      }
      __syncwarp();
      for (uint32_t q = s0 + lane; q < s1; q += 32u) v.pos2[q] = v.pos[v.cell_atoms[q]];
    }
  }
}

// Cells of sparse replicas (k_build_sparse) with at most kSortThreadMax
// members: one thread per work item sorts its cell's slots in registers
// (insertion sort) and gathers their positions; k_cellsort sorts the rest.
__global__ void __launch_bounds__(kBlock) k_cellsort_sparse(DeviceView v) {
  const uint32_t w = blockIdx.x * kBlock + threadIdx.x;
  if (w >= v.work_start[v.n_replicas]) return;
  const uint32_t r = work_replica(v, w);
  const ReplicaParams& p = v.rp[r];
  if (!p.sparse) return;
  const uint32_t c = w - v.work_start[r];
  const uint32_t s0 = v.cell_start[p.start_base + c];
  const uint32_t s1 = v.cell_start[p.start_base + c + 1];
  const uint32_t n = s1 - s0;
  if (n > kSortThreadMax) return;
  uint32_t key[kSortThreadMax];
#pragma unroll
  for (uint32_t k = 0; k < kSortThreadMax; ++k) key[k] = k < n ? v.cell_atoms[s0 + k] : 0xffffffffu;
  // Insertion sort of a fixed-size register array (compile-time indices).
#pragma unroll
  for (uint32_t a = 1; a < kSortThreadMax; ++a) {
#pragma unroll
    for (uint32_t b = a; b > 0; --b) {
      const uint32_t lo = min(key[b - 1], key[b]), hi = max(key[b - 1], key[b]);
      key[b - 1] = lo;
      key[b] = hi;
    }
  }
#pragma unroll
  for (uint32_t k = 0; k < kSortThreadMax; ++k) {
    if (k < n) {
      v.cell_atoms[s0 + k] = key[k];
      v.pos2[s0 + k] = v.pos[key[k]];
    }
  }
}

// Warp w sorts work item w (k_scan): the warps past the cells of the
// rebuilding replicas return after one load.
__global__ void __launch_bounds__(kBlock) k_cellsort(DeviceView v) {
  __shared__ uint32_t sort_keys[kBlock / 32][kSortRankMax];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t w = blockIdx.x * (kBlock / 32) + warp;
  if (w >= v.work_start[v.n_replicas]) return;  // warp-uniform
  const uint32_t r = work_replica(v, w);
  sort_cell(v, v.rp[r], w - v.work_start[r], lane, sort_keys[warp]);
}

// rebuild 5/6: physical reorder into cell order (every sort_every builds).
__device__ __forceinline__ void reorder_gather_block(const DeviceView& v, uint32_t b) {
  const uint32_t r = v.block_replica[b];
  const ReplicaState& st = v.rs[r];
  if (!st.need_rebuild || !st.reorder_now) return;
  const ReplicaParams& p = v.rp[r];
  const uint32_t k = b * kBlock + threadIdx.x;
  if (k - p.atom_begin >= p.n_atoms) return;
  const uint32_t old = v.cell_atoms[k];  // pos2[k] is pos[old] already (k_cellsort)
  v.vel2[k] = v.vel[old];
  v.img2[k] = v.img[old];
  v.tag2[k] = v.tag[old];
  v.mol2[k] = v.mol[old];
  v.cell2[k] = v.cell_of_slot[old];
}

__global__ void __launch_bounds__(kBlock) k_reorder_gather(DeviceView v) {
  for_chain_blocks<reorder_gather_block>(v);
}

__device__ __forceinline__ void reorder_commit_block(const DeviceView& v, uint32_t b) {
  const uint32_t r = v.block_replica[b];
  const ReplicaState& st = v.rs[r];
  if (!st.need_rebuild || !st.reorder_now) return;
  const ReplicaParams& p = v.rp[r];
  const uint32_t k = b * kBlock + threadIdx.x;
  if (k - p.atom_begin >= p.n_atoms) return;
  v.pos[k] = v.pos2[k];
  v.vel[k] = v.vel2[k];
  v.img[k] = v.img2[k];
  const uint32_t t = v.tag2[k];
  v.tag[k] = t;
  v.mol[k] = v.mol2[k];
  v.cell_of_slot[k] = v.cell2[k];
  v.cell_atoms[k] = k;
  v.slot_of_tag[t] = k;
}

__global__ void __launch_bounds__(kBlock) k_reorder_commit(DeviceView v) {
  for_chain_blocks<reorder_commit_block>(v);
}

// Exclusion partners of every slot, projected from tag space to slot space
// (the reference's SlotExclusionRuntime::rebuild_from_source,
// exclusions.cu:337-460, here one fixed-width row per slot).
__global__ void __launch_bounds__(kBlock)
k_project_exclusions(DeviceView v, int force_all) {
  const uint32_t b = blockIdx.x;
  const uint32_t r = v.block_replica[b];
  const ReplicaState& st = v.rs[r];
  if (!force_all && (!st.need_rebuild || !st.reorder_now)) return;
  const ReplicaParams& p = v.rp[r];
  const uint32_t k = b * kBlock + threadIdx.x;
  if (k - p.atom_begin >= p.n_atoms) return;
  const uint32_t t = v.tag[k];
  const uint32_t e0 = v.excl_off[t];
  const uint32_t e1 = v.excl_off[t + 1];
  uint32_t* row = v.excl_slot + (size_t)k * v.excl_cap;
  for (uint32_t e = 0; e < v.excl_cap; ++e) {
    row[e] = (e0 + e < e1) ? v.slot_of_tag[v.excl_tag[e0 + e]] : 0xffffffffu;
  }
}

// rebuild 7: full neighbour list over the cell stencil, reference inclusion
// rule: skip self and excluded partners, keep r^2 <= (rc+skin)^2, count
// overflow past max_neighbors.  Also captures the displacement reference.
//
// One warp per cell, the candidates on the lanes.  The stencil of the cell is
// a list of segments (contiguous runs of cell_atoms) in the reference's
// stencil order (z, y, x cells; ascending slot inside a cell); their
// concatenation is the candidate stream, walked kChunk (128) candidates at
// a time: lane l holds candidates l, 32 + l, 64 + l and 96 + l of a chunk
// as two packed pairs, all tested against one home particle per iteration
// on the packed FP32x2 pipe.  Four ballots give the accepted candidates in
// stream order; each accepted lane writes its
// entry at the home particle's count plus its rank among the accepted, so a
// particle's list order is the stream order under any schedule.  Every lane
// does useful work whatever the cell occupancy, and appends never diverge.
//
// Regular grids (every axis >= 4 cells): a stencil row of three x-cells is
// one segment (two where it wraps in x), 18 segments at most.  A cell
// reached across the periodic boundary gets one shift s = +-L for the whole
// segment and the difference is fl(fl(xi - xj) + s).  For any pair that can
// pass the search cutoff this is exactly the reference's form (fl(xi - xj),
// then fl(d -+ L) when |d| > L/2), because with >= 4 cells per axis a
// neighbour-cell pair has |xi - xj| < L/2 unless it wraps, and a wrapped one
// has |xi - xj| > L/2.  Cells away from the boundary have no shift at all.
// Small-dimension and direct grids: each of the min(n, 3)^3 stencil cells is
// a segment and the reference's minimum image is applied per pair.
constexpr int kBuildWarps = kBlock / 32;
constexpr uint32_t kMaxSegments = 27;

// ---------------------------------------------------------------------------
// Cell-tile staging of the pair-force kernel.
//
// In a staged context the list of a particle is stored in ROW q, its index in
// the cell order of the last build (cell_atoms[q] is its slot), and a
// "group" is 128 consecutive rows: the particles of k_lj_staged's block.  The
// home cells of a group are one contiguous run of cell indices; the group's
// STAGE is the union of their stencils, laid out as windows: for every home
// row (a run of cells of one x-row, at most kStageRows of them) and every one
// of its 9 stencil rows, the cells [xa - 1, xb + 2) of that row, cut in two
// where they wrap in x (or the whole row when that is shorter).  A window is
// a contiguous run of cell-order indices, so the stage holds
// pos[cell_atoms[q]] for q in every window, one after another; the force
// kernel copies it into shared memory once per step.  A list entry of a
// staged group is the neighbour's stage index (q + delta of its window); a
// group whose stage would exceed the context's capacity, or whose home cells
// span more rows, keeps slot entries and gathers positions from global
// memory instead.  The build and the force kernel derive the layout from the
// same cell_start by the same function, so they agree on it.
constexpr uint32_t kStageRows = 3;                      // home rows per group at most
constexpr uint32_t kStageWindows = 2 * 9 * kStageRows;  // 54
struct StageLayout {
  uint32_t n_win;                  // windows (0: the group keeps slot entries)
  uint32_t size;                   // stage entries
  uint32_t row_first;              // replica-local row (y + ny z) of the first home cell
  uint32_t q_first, q_end;         // rows of the group's particles
  uint32_t qbeg[kStageWindows];    // cell-order index of a window's first entry
  uint32_t base[kStageWindows];    // its stage index
  uint32_t x0[kStageWindows];      // x-range of its cells
  uint32_t x1[kStageWindows];
};

// Fills `lay` for group g (one full warp; lay is the warp's shared scratch).
// Only replicas with the staged flag and grids of >= 4 cells on every axis
// are staged: their stencil rows are distinct and their segments never wrap
// inside a window.
__device__ __forceinline__ void stage_layout(const DeviceView& v, const ReplicaParams& p,
                                             uint32_t g, uint32_t lane, uint32_t cap,
                                             StageLayout& lay) {
  const uint32_t q_lo = max(g * (uint32_t)kBlock, p.atom_begin);
  const uint32_t q_hi = min((g + 1u) * (uint32_t)kBlock, p.atom_begin + p.n_atoms);
  const uint32_t nx = p.nc[0], ny = p.nc[1], nz = p.nc[2];
  bool ok = p.staged != 0u && q_lo < q_hi && nx >= 4u && ny >= 4u && nz >= 4u;
  uint32_t cf = 0, cl = 0;
  if (ok) {
    cf = v.cell_of_slot[v.cell_atoms[q_lo]] - p.cell_begin;
    cl = v.cell_of_slot[v.cell_atoms[q_hi - 1u]] - p.cell_begin;
  }
  const uint32_t rf = cf / nx, rl = cl / nx;
  const uint32_t nsub = ok ? rl - rf + 1u : 0u;
  ok = ok && nsub <= kStageRows;
  // lane l < 9 nsub: home row rf + l / 9, stencil row l % 9 (z-major, as the
  // build walks it); two windows per lane.
  uint32_t qa0 = 0, qa1 = 0, qb0 = 0, qb1 = 0, xa0 = 0, xa1 = 0, xb0 = 0, xb1 = 0;
  if (ok && lane < 9u * nsub) {
    const uint32_t sub = lane / 9u, k = lane % 9u;
    const uint32_t row = rf + sub;
    const uint32_t y = row % ny, z = row / ny;
    const uint32_t xa = sub == 0u ? cf % nx : 0u;
    const uint32_t xb = sub + 1u == nsub ? cl % nx : nx - 1u;
    const uint32_t yy = stencil_cell(y, ny, k % 3u), zz = stencil_cell(z, nz, k / 3u);
    const uint32_t rowbase = nx * (yy + ny * zz);
    if (xb - xa + 3u >= nx) {
      xa0 = 0u, xa1 = nx;
    } else if (xa == 0u) {
      xa0 = nx - 1u, xa1 = nx, xb0 = 0u, xb1 = xb + 2u;
    } else if (xb == nx - 1u) {
      xa0 = xa - 1u, xa1 = nx, xb0 = 0u, xb1 = 1u;
    } else {
      xa0 = xa - 1u, xa1 = xb + 2u;
    }
    const uint32_t* start = v.cell_start + p.start_base;
    qa0 = start[rowbase + xa0];
    qa1 = start[rowbase + xa1];
    if (xb1 > xb0) {
      qb0 = start[rowbase + xb0];
      qb1 = start[rowbase + xb1];
    }
  }
  const uint32_t len = (qa1 - qa0) + (qb1 - qb0);
  uint32_t inc = len;
#pragma unroll
  for (uint32_t o = 1; o < 32u; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, inc, o);
    if (lane >= o) inc += t;
  }
  const uint32_t total = __shfl_sync(kFull, inc, 31);
  ok = ok && total <= cap;
  __syncwarp();
  if (lane < 9u * kStageRows) {
    const uint32_t b = inc - len;
    lay.qbeg[2 * lane] = qa0;
    lay.base[2 * lane] = b;
    lay.x0[2 * lane] = xa0;
    lay.x1[2 * lane] = xa1;
    lay.qbeg[2 * lane + 1] = qb0;
    lay.base[2 * lane + 1] = b + (qa1 - qa0);
    lay.x0[2 * lane + 1] = xb0;
    lay.x1[2 * lane + 1] = xb1;
  }
  if (lane == 0) {
    lay.n_win = ok ? 18u * nsub : 0u;
    lay.size = ok ? total : 0u;
    lay.row_first = rf;
    lay.q_first = q_lo;
    lay.q_end = q_hi;
  }
  __syncwarp();
}

struct BuildShared {
  uint32_t seg_end[kMaxSegments];  // stream offset one past the segment
  uint32_t seg_q[kMaxSegments];    // cell_atoms index of the segment's stream offset 0
  float seg_s[3][kMaxSegments];    // periodic shift of the segment (regular grids)
  float4 home_a[32];               // {x, x, y, y} of the home particles
  float4 home_b[32];               // {z, z, slot bits, 0}
  // Staged contexts: the home particles in flight belong to one group; a
  // candidate's entry is its cell-order index + delta[segment] when that
  // group is staged, else its slot.
  uint32_t delta[kMaxSegments];
  StageLayout lay;
};

enum BuildForm : int { kBuildInterior = 0, kBuildShifted = 1, kBuildMinImage = 2 };

// Candidates of one lane in a chunk: kBuildPairs pairs, pair q holding
// stream positions base + 64 q + lane (.x) and base + 64 q + 32 + lane (.y).
struct CandPair {
  uint32_t jx, jy;       // slots (0xffffffff past the stream)
  uint32_t ex, ey;       // list entries: stage indices in a staged group, else the slots
  float2 nx, ny, nz;     // minus their coordinates
  float2 sx, sy, sz;     // periodic shifts of their segments
};
constexpr int kBuildPairs = 2;
constexpr uint32_t kChunk = 64u * kBuildPairs;  // candidates per chunk

// Tests one chunk of candidates against the home particles [0, nh) and
// appends the accepted ones.  my_cnt: lane h holds home particle h's count.
template <int kCap, int kForm>
__device__ __forceinline__ void build_chunk(const DeviceView& v, const ReplicaParams& p,
                                            const BuildShared& sh, uint32_t nh, uint32_t lane,
                                            const CandPair (&c)[kBuildPairs],
                                            uint32_t& my_cnt) {
  const float cut = p.search_cut_sq;
  const uint32_t cap = p.max_neighbors;
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll 1
  for (uint32_t h = 0; h < nh; ++h) {
    const float4 ha = sh.home_a[h];
    const float4 hb = sh.home_b[h];
    const uint32_t i = __float_as_uint(hb.z);
    bool ax[kBuildPairs], ay[kBuildPairs];
    uint32_t bx[kBuildPairs], by[kBuildPairs];
    uint32_t any = 0u;
#pragma unroll
    for (int q = 0; q < kBuildPairs; ++q) {
      float2 dx, dy, dz;
      if (kForm == kBuildMinImage) {
        dx = make_float2(ref_delta(ha.x, -c[q].nx.x, p.len[0], p.half[0]),
                         ref_delta(ha.x, -c[q].nx.y, p.len[0], p.half[0]));
        dy = make_float2(ref_delta(ha.z, -c[q].ny.x, p.len[1], p.half[1]),
                         ref_delta(ha.z, -c[q].ny.y, p.len[1], p.half[1]));
        dz = make_float2(ref_delta(hb.x, -c[q].nz.x, p.len[2], p.half[2]),
                         ref_delta(hb.x, -c[q].nz.y, p.len[2], p.half[2]));
      } else {
        // fl(xi + (-xj)) is fl(xi - xj); a zero shift leaves it unchanged.
        dx = __fadd2_rn(make_float2(ha.x, ha.y), c[q].nx);
        dy = __fadd2_rn(make_float2(ha.z, ha.w), c[q].ny);
        dz = __fadd2_rn(make_float2(hb.x, hb.y), c[q].nz);
        if (kForm == kBuildShifted) {
          dx = __fadd2_rn(dx, c[q].sx);
          dy = __fadd2_rn(dy, c[q].sy);
          dz = __fadd2_rn(dz, c[q].sz);
        }
      }
      const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dx, dx, __fmul2_rn(dy, dy)));
      ax[q] = !(r2.x > cut) && c[q].jx != i;
      ay[q] = !(r2.y > cut) && c[q].jy != i;
      bx[q] = __ballot_sync(kFull, ax[q]);
      by[q] = __ballot_sync(kFull, ay[q]);
      any |= bx[q] | by[q];
    }
    if (any == 0u) continue;  // warp-uniform
    if (kCap > 0) {
      // Exclusion rows are padded with 0xffffffff after the last partner.
      const uint32_t* ex = v.excl_slot + (size_t)i * v.excl_cap;
#pragma unroll 4
      for (int e = 0; e < kCap; ++e) {
        const uint32_t xe = __ldg(ex + e);
        if (xe == 0xffffffffu) break;  // warp-uniform
#pragma unroll
        for (int q = 0; q < kBuildPairs; ++q) {
          ax[q] = ax[q] && c[q].jx != xe;
          ay[q] = ay[q] && c[q].jy != xe;
        }
      }
#pragma unroll
      for (int q = 0; q < kBuildPairs; ++q) {
        bx[q] = __ballot_sync(kFull, ax[q]);
        by[q] = __ballot_sync(kFull, ay[q]);
      }
    }
    uint32_t k = __shfl_sync(kFull, my_cnt, h);
    // The list row: the slot, or in a staged context the cell-order index.
    uint32_t* row = v.nbr + nbr_index(__float_as_uint(hb.w), 0, v.nbr_stride);
#pragma unroll
    for (int q = 0; q < kBuildPairs; ++q) {
      const uint32_t kx = k + __popc(bx[q] & lt);
      k += __popc(bx[q]);
      const uint32_t ky = k + __popc(by[q] & lt);
      k += __popc(by[q]);
      if (ax[q] && kx < cap) row[(size_t)kx * kGroup] = c[q].ex;
      if (ay[q] && ky < cap) row[(size_t)ky * kGroup] = c[q].ey;
    }
    if (lane == h) my_cnt = k;
  }
}

// The list rows of the particles of global cell g (one warp).  kByQ: the
// context lists rows by cell-order index (staged layout); a compile-time
// flag so that the slot-layout build carries none of the staging code.
template <int kCap, bool kByQ>
__device__ __forceinline__ void build_cell(const DeviceView& v, const ReplicaParams& p,
                                           ReplicaState* st, uint32_t g, uint32_t lane,
                                           BuildShared& sh) {
  if (p.sparse) return;  // built by k_build_sparse
  const uint32_t c = g - p.cell_begin;
  const uint32_t* start = v.cell_start + p.start_base;
  const uint32_t cs = start[c], ce = start[c + 1];
  if (cs == ce) return;
  const uint32_t nx = p.nc[0], ny = p.nc[1], nz = p.nc[2];
  const uint32_t cx = c % nx, cy = (c / nx) % ny, cz = c / (nx * ny);
  const bool regular = nx >= 4u && ny >= 4u && nz >= 4u;

  // Segment table: lane s describes segment s.
  uint32_t q0 = 0u, q1 = 0u;
  float shx = 0.0f, shy = 0.0f, shz = 0.0f;
  uint32_t seg_lo = 0u, seg_k = 0u;  // x of the segment's first cell, its stencil row
  if (regular) {
    if (lane < 18u) {
      const uint32_t a = lane / 6u, bb = (lane / 2u) % 3u, sg = lane & 1u;
      seg_k = 3u * a + bb;
      const uint32_t zc = stencil_cell(cz, nz, a), yc = stencil_cell(cy, ny, bb);
      shz = (cz == 0u && a == 0u) ? p.len[2] : (cz == nz - 1u && a == 2u) ? -p.len[2] : 0.0f;
      shy = (cy == 0u && bb == 0u) ? p.len[1] : (cy == ny - 1u && bb == 2u) ? -p.len[1] : 0.0f;
      // A row is [cx-1, cx+2) unless it wraps in x, where it splits in two.
      uint32_t lo = cx - 1u, hi = cx + 2u;
      bool used = sg == 0u;
      if (cx == 0u) {
        lo = sg == 0u ? nx - 1u : 0u, hi = sg == 0u ? nx : 2u, used = true;
        shx = sg == 0u ? p.len[0] : 0.0f;
      } else if (cx == nx - 1u) {
        lo = sg == 0u ? nx - 2u : 0u, hi = sg == 0u ? nx : 1u, used = true;
        shx = sg == 0u ? 0.0f : -p.len[0];
      }
      if (used) {
        const uint32_t row = nx * (yc + ny * zc);
        q0 = start[row + lo];
        q1 = start[row + hi];
      }
      seg_lo = lo;
    }
  } else {
    const uint32_t sxn = min(nx, 3u), syn = min(ny, 3u), szn = min(nz, 3u);
    if (lane < sxn * syn * szn) {
      const uint32_t k = lane % sxn, bb = (lane / sxn) % syn, a = lane / (sxn * syn);
      const uint32_t lc = stencil_cell(cx, nx, k) +
                          nx * (stencil_cell(cy, ny, bb) + ny * stencil_cell(cz, nz, a));
      q0 = start[lc];
      q1 = start[lc + 1];
    }
  }
  uint32_t end = q1 - q0;  // inclusive scan of the segment lengths
#pragma unroll
  for (uint32_t o = 1; o < 32u; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, end, o);
    if (lane >= o) end += t;
  }
  const uint32_t total = __shfl_sync(kFull, end, 31);
  __syncwarp();
  if (lane < kMaxSegments) {
    sh.seg_end[lane] = end;
    sh.seg_q[lane] = q0 - (end - (q1 - q0));
    sh.seg_s[0][lane] = shx;
    sh.seg_s[1][lane] = shy;
    sh.seg_s[2][lane] = shz;
  }
  const int form = !regular ? kBuildMinImage
                   : (cx == 0u || cy == 0u || cz == 0u || cx == nx - 1u || cy == ny - 1u ||
                      cz == nz - 1u)
                       ? kBuildShifted
                       : kBuildInterior;
  const uint32_t nseg = regular ? 18u : kMaxSegments;
  bool any_overflow = false;
  constexpr bool by_q = kByQ;
  const bool staged_replica = by_q && p.staged != 0u && regular;

  // In a staged context the home particles in flight never span two groups
  // (128 cell-order rows), so one stage layout serves all of them.
  for (uint32_t i0 = cs, i1 = 0; i0 < ce; i0 = i1) {
    i1 = min(i0 + 32u, ce);
    if (staged_replica) i1 = min(i1, (i0 / (uint32_t)kBlock + 1u) * (uint32_t)kBlock);
    const uint32_t nh = i1 - i0;
    bool staged_group = false;
    if (staged_replica) {
      stage_layout(v, p, i0 / (uint32_t)kBlock, lane, v.stage_cap, sh.lay);
      staged_group = sh.lay.n_win != 0u;
      if (staged_group && lane < 18u) {
        const uint32_t w0 = 2u * (((cy + ny * cz) - sh.lay.row_first) * 9u + seg_k);
        const uint32_t w = (sh.lay.x0[w0] <= seg_lo && seg_lo < sh.lay.x1[w0]) ? w0 : w0 + 1u;
        sh.delta[lane] = sh.lay.base[w] - sh.lay.qbeg[w];
      }
    }
    uint32_t i = 0u;
    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncwarp();
    if (lane < nh) {
      i = v.cell_atoms[i0 + lane];
      xi = v.pos2[i0 + lane];
      sh.home_a[lane] = make_float4(xi.x, xi.x, xi.y, xi.y);
      sh.home_b[lane] = make_float4(xi.z, xi.z, __uint_as_float(i),
                                    __uint_as_float(by_q ? i0 + lane : i));
    }
    __syncwarp();
    uint32_t my_cnt = 0u;
    uint32_t seg[2 * kBuildPairs] = {};  // segment walk of this lane's stream positions
    for (uint32_t base = 0; base < total; base += kChunk) {
      CandPair c[kBuildPairs];
#pragma unroll
      for (int t = 0; t < 2 * kBuildPairs; ++t) {
        const uint32_t u = base + 32u * t + lane;
        while (seg[t] < nseg && u >= sh.seg_end[seg[t]]) ++seg[t];
        // Past the stream: an infinite coordinate fails every distance test
        // against a finite home particle.  Its slot and entry are the far
        // particle's (pos[n_slots], or the stage's last entry), so even a
        // home particle with non-finite coordinates, which accepts every
        // candidate (r^2 NaN is not above the cutoff, the reference's rule),
        // lists only valid indices.
        uint32_t j = v.n_slots;
        float4 x = make_float4(INFINITY, 0.f, 0.f, 0.f);
        const uint32_t st = min(seg[t], kMaxSegments - 1u);
        const uint32_t qc = sh.seg_q[st] + u;
        uint32_t e = staged_group ? sh.lay.size : v.n_slots;
        if (u < total) {
          j = v.cell_atoms[qc];
          x = v.pos2[qc];
          e = staged_group ? qc + sh.delta[st] : j;
        }
        const float sx = form == kBuildShifted ? sh.seg_s[0][st] : 0.f;
        const float sy = form == kBuildShifted ? sh.seg_s[1][st] : 0.f;
        const float sz = form == kBuildShifted ? sh.seg_s[2][st] : 0.f;
        CandPair& cp = c[t >> 1];
        if ((t & 1) == 0) {
          cp.jx = j, cp.ex = e, cp.nx.x = -x.x, cp.ny.x = -x.y, cp.nz.x = -x.z;
          cp.sx.x = sx, cp.sy.x = sy, cp.sz.x = sz;
        } else {
          cp.jy = j, cp.ey = e, cp.nx.y = -x.x, cp.ny.y = -x.y, cp.nz.y = -x.z;
          cp.sx.y = sx, cp.sy.y = sy, cp.sz.y = sz;
        }
      }
      if (form == kBuildInterior) {
        build_chunk<kCap, kBuildInterior>(v, p, sh, nh, lane, c, my_cnt);
      } else if (form == kBuildShifted) {
        build_chunk<kCap, kBuildShifted>(v, p, sh, nh, lane, c, my_cnt);
      } else {
        build_chunk<kCap, kBuildMinImage>(v, p, sh, nh, lane, c, my_cnt);
      }
    }
    if (lane < nh) {
      v.nbr_count[by_q ? i0 + lane : i] = min(my_cnt, p.max_neighbors);
      v.ref_pos[i] = xi;
      v.ref_img[i] = v.img[i];
      v.cross[i] = 0u;
    }
    any_overflow |= lane < nh && my_cnt > p.max_neighbors;
  }
  if (__any_sync(kFull, any_overflow) && lane == 0) atomicOr(&st->status, kStatusNeighborOverflow);
}

// Warp w builds the lists of work item w (k_scan): the warps past the cells
// of the rebuilding replicas return after one load.
template <int kCap, bool kByQ>
__global__ void __launch_bounds__(kBlock, 7) k_build(DeviceView v) {
  __shared__ BuildShared sh[kBuildWarps];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t w = blockIdx.x * kBuildWarps + warp;
  if (w >= v.work_start[v.n_replicas]) return;  // warp-uniform
  const uint32_t r = work_replica(v, w);
  const ReplicaParams& p = v.rp[r];
  build_cell<kCap, kByQ>(v, p, &v.rs[r], p.cell_begin + (w - v.work_start[r]), lane, sh[warp]);
}

// The same lists, one thread per particle, for replicas whose cells hold a
// few particles each (a bead-spring melt at WCA range: ~2.4 per cell), where
// a warp per cell leaves most lanes idle and spends its time on the segment
// table.  Thread q takes the particle at cell-order index q, walks the
// stencil segments of its cell in build_cell's order (z, y rows; the x run
// of a row, split in two where it wraps; ascending slot inside a cell) and
// applies build_cell's float expressions, inclusion rule and entry encoding,
// so the lists (order included) are the ones k_build writes.  A block is 128
// consecutive cell-order rows: one stage group in a staged context.  kByQ
// as for k_build.
template <int kCap, bool kByQ>
__global__ void __launch_bounds__(kBlock) k_build_sparse(DeviceView v) {
  __shared__ StageLayout lay;
  const uint32_t b = blockIdx.x;
  const uint32_t r = v.block_replica[b];
  const ReplicaParams& p = v.rp[r];
  ReplicaState* st = &v.rs[r];
  if (!p.sparse || !st->need_rebuild) return;  // block-uniform
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t nx = p.nc[0], ny = p.nc[1], nz = p.nc[2];
  const bool regular = nx >= 4u && ny >= 4u && nz >= 4u;
  constexpr bool by_q = kByQ;
  const bool staged_replica = by_q && p.staged != 0u && regular;
  if (staged_replica) {
    if (warp == 0) stage_layout(v, p, b, lane, v.stage_cap, lay);
    __syncthreads();
  }
  const bool staged_group = staged_replica && lay.n_win != 0u;
  const uint32_t q = b * kBlock + threadIdx.x;
  if (q - p.atom_begin >= p.n_atoms) return;
  const uint32_t i = v.cell_atoms[q];
  const float4 xi = v.pos2[q];
  const uint32_t c = v.cell_of_slot[i] - p.cell_begin;
  const uint32_t cx = c % nx, cy = (c / nx) % ny, cz = c / (nx * ny);
  const uint32_t* start = v.cell_start + p.start_base;
  const int form = !regular ? kBuildMinImage
                   : (cx == 0u || cy == 0u || cz == 0u || cx == nx - 1u || cy == ny - 1u ||
                      cz == nz - 1u)
                       ? kBuildShifted
                       : kBuildInterior;
  const float cut = p.search_cut_sq;
  const uint32_t cap = p.max_neighbors;
  uint32_t ex[kCap > 0 ? kCap : 1];
  if (kCap > 0) {
    const uint32_t* er = v.excl_slot + (size_t)i * v.excl_cap;
#pragma unroll
    for (int e = 0; e < kCap; ++e) ex[e] = er[e];
  }
  uint32_t* row = v.nbr + nbr_index(by_q ? q : i, 0, v.nbr_stride);
  uint32_t cnt = 0u;
  // One segment: cell-order run [q0, q1), periodic shift (sx, sy, sz) for the
  // shifted form, entry offset `delta` (stage index = q + delta) in a staged
  // group.
  auto walk = [&](uint32_t q0, uint32_t q1, float sx, float sy, float sz, uint32_t delta) {
    for (uint32_t qc = q0; qc < q1; ++qc) {
      const uint32_t j = v.cell_atoms[qc];
      const float4 x = v.pos2[qc];
      float dx, dy, dz;
      if (form == kBuildMinImage) {
        dx = ref_delta(xi.x, x.x, p.len[0], p.half[0]);
        dy = ref_delta(xi.y, x.y, p.len[1], p.half[1]);
        dz = ref_delta(xi.z, x.z, p.len[2], p.half[2]);
      } else {
        dx = __fsub_rn(xi.x, x.x);
        dy = __fsub_rn(xi.y, x.y);
        dz = __fsub_rn(xi.z, x.z);
        if (form == kBuildShifted) {
          dx = __fadd_rn(dx, sx);
          dy = __fadd_rn(dy, sy);
          dz = __fadd_rn(dz, sz);
        }
      }
      bool ok = !(norm2(dx, dy, dz) > cut) && j != i;
      if (kCap > 0) {
#pragma unroll
        for (int e = 0; e < kCap; ++e) ok = ok && j != ex[e];
      }
      if (ok) {
        if (cnt < cap) row[(size_t)cnt * kGroup] = staged_group ? qc + delta : j;
        ++cnt;
      }
    }
  };
  if (regular) {
    for (uint32_t a = 0; a < 3u; ++a) {
      const uint32_t zc = stencil_cell(cz, nz, a);
      const float shz = (cz == 0u && a == 0u) ? p.len[2] : (cz == nz - 1u && a == 2u) ? -p.len[2] : 0.0f;
      for (uint32_t bb = 0; bb < 3u; ++bb) {
        const uint32_t yc = stencil_cell(cy, ny, bb);
        const float shy = (cy == 0u && bb == 0u) ? p.len[1] : (cy == ny - 1u && bb == 2u) ? -p.len[1] : 0.0f;
        const uint32_t rowbase = nx * (yc + ny * zc);
        const uint32_t k = 3u * a + bb;
        for (uint32_t sg = 0; sg < 2u; ++sg) {
          uint32_t lo = cx - 1u, hi = cx + 2u;
          float shx = 0.0f;
          bool used = sg == 0u;
          if (cx == 0u) {
            lo = sg == 0u ? nx - 1u : 0u, hi = sg == 0u ? nx : 2u, used = true;
            shx = sg == 0u ? p.len[0] : 0.0f;
          } else if (cx == nx - 1u) {
            lo = sg == 0u ? nx - 2u : 0u, hi = sg == 0u ? nx : 1u, used = true;
            shx = sg == 0u ? 0.0f : -p.len[0];
          }
          if (!used) continue;
          uint32_t delta = 0u;
          if (staged_group) {
            const uint32_t w0 = 2u * (((cy + ny * cz) - lay.row_first) * 9u + k);
            const uint32_t w = (lay.x0[w0] <= lo && lo < lay.x1[w0]) ? w0 : w0 + 1u;
            delta = lay.base[w] - lay.qbeg[w];
          }
          walk(start[rowbase + lo], start[rowbase + hi], shx, shy, shz, delta);
        }
      }
    }
  } else {
    const uint32_t sxn = min(nx, 3u), syn = min(ny, 3u), szn = min(nz, 3u);
    for (uint32_t a = 0; a < szn; ++a) {
      for (uint32_t bb = 0; bb < syn; ++bb) {
        for (uint32_t k = 0; k < sxn; ++k) {
          const uint32_t lc = stencil_cell(cx, nx, k) +
                              nx * (stencil_cell(cy, ny, bb) + ny * stencil_cell(cz, nz, a));
          walk(start[lc], start[lc + 1], 0.0f, 0.0f, 0.0f, 0u);
        }
      }
    }
  }
  v.nbr_count[by_q ? q : i] = min(cnt, p.max_neighbors);
  v.ref_pos[i] = xi;
  v.ref_img[i] = v.img[i];
  v.cross[i] = 0u;
  if (cnt > p.max_neighbors) atomicOr(&st->status, kStatusNeighborOverflow);
}

// ---------------------------------------------------------------------------
// Second half-kick of a step, shared by k_post and by the force kernels that
// finish a step themselves (see k_post).
enum ForceMode : int {
  kForcePlain = 0,        // forces only
  kForceClamp = 1,        // forces on r^2 clamped to >= 0.49 sigma^2 (descent)
  kForcePost = 2,         // forces, then the second half-kick
  kForcePostKinetic = 3,  // forces, kick and the kinetic-energy total
};

// Kick of one slot with its final force, from its velocity vm as loaded
// before; returns its kinetic energy.
template <bool kKick, bool kKinetic>
__device__ __forceinline__ double post_slot_vm(const DeviceView& v, const ReplicaParams& p,
                                               ReplicaState* st, uint32_t i, bool real,
                                               float4 vm, float fx, float fy, float fz) {
  double ke = 0.0;
  if (real) {
    if (kKick) {
      const float h = __fdiv_rn(__fmul_rn(0.5f, p.dt), vm.w);
      vm.x = __fmaf_rn(h, fx, vm.x);
      vm.y = __fmaf_rn(h, fy, vm.y);
      vm.z = __fmaf_rn(h, fz, vm.z);
      v.vel[i] = vm;
      if (!isfinite(vm.x + vm.y + vm.z)) atomicOr(&st->status, kStatusNonFinite);
    }
    if (kKinetic) {
      const double vx = vm.x, vy = vm.y, vz = vm.z;
      ke = 0.5 * (double)vm.w * (vx * vx + vy * vy + vz * vz);
    }
  }
  return ke;
}

template <bool kKick, bool kKinetic>
__device__ __forceinline__ double post_slot(const DeviceView& v, const ReplicaParams& p,
                                            ReplicaState* st, uint32_t i, bool real,
                                            float fx, float fy, float fz) {
  const float4 vm = real ? v.vel[i] : make_float4(0.f, 0.f, 0.f, 1.f);
  return post_slot_vm<kKick, kKinetic>(v, p, st, i, real, vm, fx, fy, fz);
}

// The kernel that kicks (k_post, or the last force kernel when the kick is
// fused) sums each warp's kinetic energies in fixed point and adds the warp's
// total into one of kKeBuckets buckets of its replica (warp index modulo
// kKeBuckets): no block barrier, so a warp retires as soon as it is done,
// and few warps share a bucket.  Integer sums do not depend on order, so the
// total is the same bits whatever the schedule.  k_post_finish, one block
// per replica, then sums and empties that replica's buckets and does the
// per-replica epilogue: Berendsen lambda for the next step, step counter,
// observables.
template <bool kKinetic>
__device__ __forceinline__ void post_partial(const DeviceView& v, ReplicaState* st, uint32_t r,
                                             bool real, double ke) {
  if (!kKinetic) return;
  const Fixed f = real ? to_fixed(ke, &st->status) : Fixed{0, 0};
  long long a = f.whole, c = f.frac;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(kFull, a, o);
    c += __shfl_down_sync(kFull, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    unsigned long long* bucket = reinterpret_cast<unsigned long long*>(v.ke_part) +
                                 2 * ((size_t)r * kKeBuckets + warp % kKeBuckets);
    if (a != 0) atomicAdd(bucket, static_cast<unsigned long long>(a));
    if (c != 0) atomicAdd(bucket + 1, static_cast<unsigned long long>(c));
  }
}

// Same, one bucket add per block (k_post: a short streaming kernel where the
// block barrier costs little and fewer adds contend for the buckets).
template <bool kKinetic>
__device__ __forceinline__ void post_partial_block(const DeviceView& v, ReplicaState* st,
                                                   uint32_t r, bool real, double ke) {
  if (!kKinetic) return;
  __shared__ long long part[2][kBlock / 32];
  const Fixed f = real ? to_fixed(ke, &st->status) : Fixed{0, 0};
  long long a = f.whole, c = f.frac;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(kFull, a, o);
    c += __shfl_down_sync(kFull, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    part[0][threadIdx.x >> 5] = a;
    part[1][threadIdx.x >> 5] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long sa = 0, sc = 0;
    for (int w = 0; w < kBlock / 32; ++w) {
      sa += part[0][w];
      sc += part[1][w];
    }
    unsigned long long* bucket = reinterpret_cast<unsigned long long*>(v.ke_part) +
                                 2 * ((size_t)r * kKeBuckets + blockIdx.x % kKeBuckets);
    if (sa != 0) atomicAdd(bucket, static_cast<unsigned long long>(sa));
    if (sc != 0) atomicAdd(bucket + 1, static_cast<unsigned long long>(sc));
  }
}

constexpr int kFinishThreads = 128;
static_assert(kKeBuckets <= (uint32_t)kFinishThreads, "one finish thread per bucket");

template <bool kKick, bool kObs, bool kKinetic>
__global__ void __launch_bounds__(kFinishThreads) k_post_finish(DeviceView v) {
  wait_prior_grid();
  const uint32_t r = blockIdx.x;
  const ReplicaParams& p = v.rp[r];
  ReplicaState* st = &v.rs[r];
  __shared__ long long part[2][kFinishThreads / 32];
  long long a = 0, c = 0;
  if (kKinetic) {
    if (threadIdx.x < kKeBuckets) {
      longlong2* bucket = reinterpret_cast<longlong2*>(v.ke_part) + (size_t)r * kKeBuckets +
                          threadIdx.x;
      const longlong2 q = *bucket;
      *bucket = make_longlong2(0, 0);
      a = q.x;
      c = q.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(kFull, a, o);
      c += __shfl_down_sync(kFull, c, o);
    }
    if ((threadIdx.x & 31) == 0) {
      part[0][threadIdx.x >> 5] = a;
      part[1][threadIdx.x >> 5] = c;
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  double kin = 0.0;
  if (kKinetic) {
    long long sa = 0, sc = 0;
    for (int w = 0; w < kFinishThreads / 32; ++w) {
      sa += part[0][w];
      sc += part[1][w];
    }
    kin = from_fixed(sa, sc);
  }
  double lam = 1.0;
  if (kKick && kKinetic && p.thermostat == 1 && kin > 0.0 && p.dof > 0.0) {
    const double current = 2.0 * kin / p.dof;
    const double arg = 1.0 + ((double)p.dt / p.tau) * (p.kt_target / current - 1.0);
    lam = sqrt(arg > 0.0 ? arg : 0.0);
  }
  if (kKick) {
    st->lambda = lam;
    st->step += 1ull;
  }
  if (kKinetic) st->last_kinetic = kin;
  if (kObs) {
    ReplicaObs o;
    o.step = st->step;
    o.pair_pe = take_total(st, kAccPair);
    o.bond_pe = take_total(st, kAccBond);
    o.angle_pe = take_total(st, kAccAngle);
    o.dihedral_pe = take_total(st, kAccDihedral);
    o.virial = take_total(st, kAccVirial);
    o.ke_pre = kin;
    o.lambda = lam;
    o.builds = st->builds;
    o.dangerous = st->dangerous;
    o.status = st->status;
    o.pad = 0;
    v.obs[r] = o;
  }
}

// ---------------------------------------------------------------------------
// LJ pair forces over the full list (each pair evaluated from both ends, no
// atomics).  FP32 pair arithmetic; per-slot energy and virial are converted to
// fixed point once per slot and reduced per block.
//
// kTpa threads share one particle (threads-per-atom 1, 2 or 4, chosen by the
// engine's autotuner): thread `sub` takes list entries k = sub, sub + kTpa, ...
// Whatever kTpa, a particle's force is summed in one canonical order: four
// partial sums by k mod 4, each in ascending k, combined as
// (s0 + s1) + (s2 + s3).  So every kTpa gives the same bits and the tuning
// choice never changes a result.
template <int kTpa>
struct LjAcc {
  // kTpa 1: a[0] = (s0, s1), a[1] = (s2, s3); kTpa 2: a[0] = (s_sub, s_sub+2);
  // kTpa 4: a[0].x = s_sub.
  float2 a[kTpa == 1 ? 2 : 1];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int c = 0; c < (kTpa == 1 ? 2 : 1); ++c) a[c] = make_float2(0.f, 0.f);
  }
  // Adds the packed contributions of own entries 2h and 2h + 1 of a batch.
  __device__ __forceinline__ void add_fma(uint32_t h, float2 s, float2 d) {
    if (kTpa == 1) {
      a[h & 1u] = __ffma2_rn(s, d, a[h & 1u]);
    } else if (kTpa == 2) {
      a[0] = __ffma2_rn(s, d, a[0]);
    } else {
      a[0].x = __fmaf_rn(s.x, d.x, a[0].x);
      a[0].x = __fmaf_rn(s.y, d.y, a[0].x);
    }
  }
  __device__ __forceinline__ void add(uint32_t h, float2 t) {
    if (kTpa == 1) {
      a[h & 1u] = __fadd2_rn(a[h & 1u], t);
    } else if (kTpa == 2) {
      a[0] = __fadd2_rn(a[0], t);
    } else {
      a[0].x = __fadd_rn(a[0].x, t.x);
      a[0].x = __fadd_rn(a[0].x, t.y);
    }
  }
  // (s0 + s1) + (s2 + s3); the threads of one particle are adjacent lanes.
  __device__ __forceinline__ float total() const {
    if (kTpa == 1) return __fadd_rn(__fadd_rn(a[0].x, a[0].y), __fadd_rn(a[1].x, a[1].y));
    if (kTpa == 2) {
      const float px = __shfl_xor_sync(kFull, a[0].x, 1);
      const float py = __shfl_xor_sync(kFull, a[0].y, 1);
      return __fadd_rn(__fadd_rn(a[0].x, px), __fadd_rn(a[0].y, py));
    }
    const float pair = __fadd_rn(a[0].x, __shfl_xor_sync(kFull, a[0].x, 1));
    return __fadd_rn(pair, __shfl_xor_sync(kFull, pair, 2));
  }
};

// A neighbour-list entry: streamed (evict-first in L1) or not allocated in
// L1 at all (kNoL1), so the list stream does not displace gathered positions.
template <bool kNoL1>
__device__ __forceinline__ uint32_t list_load(const uint32_t* p) {
  if (kNoL1) {
    uint32_t v;
    asm volatile("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
  }
  return __ldcs(p);
}

// LJ coefficients of two pairs as packed pairs.  kNt = 1 (every replica has
// one particle type): the row is held in registers and already packed;
// kNt = 2: the particle's two-entry row in registers, selected by the
// neighbour's type; kNt = 0: any table, read from shared memory.
struct PairCoeff2 {
  float2 sigma2, eps24, eps4, neg_shift;
};

template <int kNt>
struct CoeffRow {
  const LjCoeff* row;
  LjCoeff r0, r1;
  PairCoeff2 one;
  __device__ __forceinline__ void init(const LjCoeff* table_row) {
    row = table_row;
    if (kNt >= 1) r0 = table_row[0];
    if (kNt == 2) r1 = table_row[1];
    if (kNt == 1) {
      one.sigma2 = make_float2(r0.sigma2, r0.sigma2);
      one.eps24 = make_float2(r0.eps24, r0.eps24);
      one.eps4 = make_float2(r0.eps4, r0.eps4);
      one.neg_shift = make_float2(-r0.shift, -r0.shift);
    }
  }
  __device__ __forceinline__ PairCoeff2 get(float w0, float w1) const {
    if (kNt == 1) return one;
    PairCoeff2 c;
    if (kNt == 2) {
      // The neighbour's type t is 0 or 1, so bits(r0) + t (bits(r1) - bits(r0))
      // picks the entry exactly, one integer multiply-add per value.
      const int t0 = __float_as_int(w0), t1 = __float_as_int(w1);
      auto pick = [](int t, float a, float b) {
        return __int_as_float(__float_as_int(a) + t * (__float_as_int(b) - __float_as_int(a)));
      };
      c.sigma2 = make_float2(pick(t0, r0.sigma2, r1.sigma2), pick(t1, r0.sigma2, r1.sigma2));
      c.eps24 = make_float2(pick(t0, r0.eps24, r1.eps24), pick(t1, r0.eps24, r1.eps24));
      c.eps4 = make_float2(pick(t0, r0.eps4, r1.eps4), pick(t1, r0.eps4, r1.eps4));
      c.neg_shift = make_float2(-pick(t0, r0.shift, r1.shift), -pick(t1, r0.shift, r1.shift));
      return c;
    }
    const LjCoeff c0 = row[__float_as_int(w0)];
    const LjCoeff c1 = row[__float_as_int(w1)];
    c.sigma2 = make_float2(c0.sigma2, c1.sigma2);
    c.eps24 = make_float2(c0.eps24, c1.eps24);
    c.eps4 = make_float2(c0.eps4, c1.eps4);
    c.neg_shift = make_float2(-c0.shift, -c1.shift);
    return c;
  }
};

// The pair loop of k_lj / k_lj_staged for one particle.  kFar = false drops
// the straddling-pair test: valid for warps whose particles all lie at least
// rc inside every face, where no pair within rc can straddle the boundary.
// The neighbour positions come from `src`: the global positions (list
// entries are slots, padding entries the far particle at n_slots) or, with
// kStage, a group's stage in shared memory (entries are stage indices, the
// far particle at the end of the stage); `row` is the particle's list row and
// `pad` the index of the far particle.
template <bool kObs, bool kClamp, int kTpa, int kUnroll, bool kNoL1, bool kFar, int kNt,
          bool kStage = false>
__device__ __forceinline__ void lj_pairs(const DeviceView& v, const ReplicaParams& p,
                                         const CoeffRow<kNt>& coeff, float4 xi, uint32_t row,
                                         const float4* src, uint32_t pad,
                                         uint32_t sub, uint32_t n, uint32_t n_warp, float rc2,
                                         float half_min_sq, LjAcc<kTpa>& ax, LjAcc<kTpa>& ay,
                                         LjAcc<kTpa>& az, LjAcc<kTpa>& ae, LjAcc<kTpa>& aw) {
  const float2 xi2x = make_float2(xi.x, xi.x);
  const float2 xi2y = make_float2(xi.y, xi.y);
  const float2 xi2z = make_float2(xi.z, xi.z);
  const uint32_t* list = v.nbr + nbr_index(row, 0, v.nbr_stride) + sub * kGroup;
  // Software-pipelined over batches of kUnroll (4 or 8) own entries: all
  // list loads of a batch are issued, then all position gathers, then the
  // arithmetic, so a warp keeps kUnroll independent misses in flight
  // instead of one (8: more misses in flight, 4: fewer registers and more
  // resident warps).  The list is streamed (evict-first) so the positions
  // stay in L2.
  // The list entries of the next batch are requested before the arithmetic
  // of the current one, so the (HBM) list latency overlaps it and only the
  // (mostly L1/L2) position gathers stay on the critical path.  kNoL1 loads
  // list entries without allocating L1 lines, leaving L1 to the gathers.
  constexpr uint32_t kStep = kUnroll * kTpa;
  uint32_t jn[kUnroll];
#pragma unroll
  for (uint32_t u = 0; u < kUnroll; ++u) {
    const uint32_t k = u * kTpa + sub;
    jn[u] = k < n ? list_load<kNoL1>(list + (size_t)(u * kTpa) * kGroup) : pad;
  }
  for (uint32_t k0 = 0; k0 < n_warp; k0 += kStep) {
    uint32_t j[kUnroll];
#pragma unroll
    for (uint32_t u = 0; u < kUnroll; ++u) j[u] = jn[u];
    float4 xj[kUnroll];
#pragma unroll
    for (uint32_t u = 0; u < kUnroll; ++u) xj[u] = kStage ? src[j[u]] : __ldg(&src[j[u]]);
#pragma unroll
    for (uint32_t u = 0; u < kUnroll; ++u) {
      const uint32_t k = k0 + kStep + u * kTpa + sub;
      jn[u] = k < n ? list_load<kNoL1>(list + (size_t)(k0 + kStep + u * kTpa) * kGroup)
                    : pad;
    }
    // Own entries 2h and 2h+1 of the batch run through the packed FP32x2
    // pipe of sm_100 (__fadd2_rn / __fmul2_rn / __ffma2_rn round each lane
    // exactly as the scalar operation would).  Pairs beyond the cutoff and
    // padding entries get a zero force scale rather than a branch.
#pragma unroll
    for (uint32_t h = 0; h < kUnroll / 2; ++h) {
      const uint32_t u0 = 2 * h, u1 = 2 * h + 1;
      float2 dx = __fadd2_rn(xi2x, make_float2(-xj[u0].x, -xj[u1].x));
      float2 dy = __fadd2_rn(xi2y, make_float2(-xj[u0].y, -xj[u1].y));
      float2 dz = __fadd2_rn(xi2z, make_float2(-xj[u0].z, -xj[u1].z));
      float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dx, dx, __fmul2_rn(dy, dy)));
      // Plain differences are already the once-rounded exact values unless
      // the pair straddles the periodic boundary, which needs r^2 above
      // (L_min/2)^2; only then (warp-uniform branch) recompute that pair
      // with the exactly rounded minimum image.
      const bool far0 = r2.x >= half_min_sq && r2.x < kFarR2;
      const bool far1 = r2.y >= half_min_sq && r2.y < kFarR2;
      if (kFar && __any_sync(kFull, far0 || far1)) {
        // Both pairs at once through the packed pipe, each lane rounded
        // exactly as acc_delta / norm2 round it; pairs that are not far keep
        // their plain differences.
        dx = acc_delta2(dx, xi2x, make_float2(-xj[u0].x, -xj[u1].x), p.len[0], p.half[0],
                        far0, far1);
        dy = acc_delta2(dy, xi2y, make_float2(-xj[u0].y, -xj[u1].y), p.len[1], p.half[1],
                        far0, far1);
        dz = acc_delta2(dz, xi2z, make_float2(-xj[u0].z, -xj[u1].z), p.len[2], p.half[2],
                        far0, far1);
        const float2 r2f = __ffma2_rn(dz, dz, __ffma2_rn(dx, dx, __fmul2_rn(dy, dy)));
        r2 = make_float2(far0 ? r2f.x : r2.x, far1 ? r2f.y : r2.y);
      }
      // Entries past the particle's count are the far particle: r^2 > rc^2.
      const bool in0 = r2.x < rc2;
      const bool in1 = r2.y < rc2;
      const PairCoeff2 c = coeff.get(xj[u0].w, xj[u1].w);
      // Out-of-range pairs get r^2 = 1e30: every power of sigma^2/r^2 then
      // underflows to 0, so their force scale is exactly 0 without a select
      // (the energy, needed only with observables, is masked explicitly).
      float2 rr = make_float2(in0 ? r2.x : 1e30f, in1 ? r2.y : 1e30f);
      if (kClamp) {
        rr.x = fmaxf(rr.x, 0.49f * c.sigma2.x);
        rr.y = fmaxf(rr.y, 0.49f * c.sigma2.y);
      }
      const float2 inv = make_float2(__fdividef(1.0f, rr.x), __fdividef(1.0f, rr.y));
      const float2 sr2 = __fmul2_rn(c.sigma2, inv);
      const float2 sr6 = __fmul2_rn(__fmul2_rn(sr2, sr2), sr2);
      const float2 sr12 = __fmul2_rn(sr6, sr6);
      const float2 neg6 = make_float2(-sr6.x, -sr6.y);
      const float2 g = __ffma2_rn(make_float2(2.0f, 2.0f), sr12, neg6);
      float2 fs = __fmul2_rn(__fmul2_rn(c.eps24, inv), g);
      ax.add_fma(h, fs, dx);
      ay.add_fma(h, fs, dy);
      az.add_fma(h, fs, dz);
      if (kObs) {
        const float2 ep = __ffma2_rn(c.eps4, __fadd2_rn(sr12, neg6), c.neg_shift);
        ae.add(h, make_float2(in0 ? ep.x : 0.0f, in1 ? ep.y : 0.0f));
        aw.add_fma(h, fs, rr);
      }
    }
  }
}

template <bool kObs, int kMode, int kTpa, int kUnroll, bool kNoL1, int kNt>
__global__ void __launch_bounds__(kBlock) k_lj(DeviceView v) {
  constexpr bool kClamp = kMode == kForceClamp;
  constexpr bool kPost = kMode >= kForcePost;
  constexpr bool kKinetic = kMode == kForcePostKinetic || (kPost && kObs);
  constexpr uint32_t kAtoms = kBlock / kTpa;  // particles per block
  const uint32_t sb = blockIdx.x / kTpa;      // 128-slot block of the particles
  const uint32_t r = v.block_replica[sb];
  const ReplicaParams& p = v.rp[r];
  __shared__ LjCoeff table[kMaxTypes * kMaxTypes];
  const int nt = p.n_types;
  for (int t = threadIdx.x; t < nt * nt; t += kBlock) table[t] = v.lj[p.lj_offset + t];
  __syncthreads();

  const uint32_t sub = threadIdx.x % kTpa;
  const uint32_t i = sb * kBlock + (blockIdx.x % kTpa) * kAtoms + threadIdx.x / kTpa;
  const bool real = (i - p.atom_begin) < p.n_atoms;
  LjAcc<kTpa> ax, ay, az, ae, aw;
  float4 vm_kick = make_float4(0.f, 0.f, 0.f, 1.f);
  ax.zero();
  ay.zero();
  az.zero();
  ae.zero();
  aw.zero();
  {
    // Every lane of the warp (padding lanes included, with n = 0) runs the
    // same number of batches, so the warp votes below are convergent.
    const float4 xi = v.pos[i];
    // With the kick fused, the velocity is requested before the pair loop so
    // its latency is hidden behind it.
    if (kPost) vm_kick = (real && sub == 0u) ? v.vel[i] : make_float4(0.f, 0.f, 0.f, 1.f);
    CoeffRow<kNt> coeff;
    coeff.init(table + __float_as_int(xi.w) * nt);
    const uint32_t n = real ? v.nbr_count[i] : 0u;
    const uint32_t n_warp = __reduce_max_sync(kFull, n);
    const float rc2 = p.force_cut_sq;
    const float hmin = fminf(p.half[0], fminf(p.half[1], p.half[2]));
    const float half_min_sq = hmin * hmin;
    // A warp whose particles all sit at least rc (with a margin) inside
    // every face has no pair within rc that straddles the boundary: its plain
    // differences are the exactly rounded minimum images, so it runs the loop
    // without the straddling test (same bits either way).
    const float rcm = 1.001f * sqrtf(rc2) + 1e-6f * fmaxf(p.len[0], fmaxf(p.len[1], p.len[2]));
    const bool inside = !real ||
        (xi.x - p.lo[0] >= rcm && p.lo[0] + p.len[0] - xi.x > rcm &&
         xi.y - p.lo[1] >= rcm && p.lo[1] + p.len[1] - xi.y > rcm &&
         xi.z - p.lo[2] >= rcm && p.lo[2] + p.len[2] - xi.z > rcm);
    if (__all_sync(kFull, inside)) {
      lj_pairs<kObs, kClamp, kTpa, kUnroll, kNoL1, false, kNt>(
          v, p, coeff, xi, i, v.pos, v.n_slots, sub, n, n_warp, rc2, half_min_sq, ax, ay, az,
          ae, aw);
    } else {
      lj_pairs<kObs, kClamp, kTpa, kUnroll, kNoL1, true, kNt>(
          v, p, coeff, xi, i, v.pos, v.n_slots, sub, n, n_warp, rc2, half_min_sq, ax, ay, az,
          ae, aw);
    }
  }
  const float fx = ax.total(), fy = ay.total(), fz = az.total();
  const bool owner = real && sub == 0u;
  if (sub == 0u) v.force[i] = make_float4(fx, fy, fz, 0.f);
  ReplicaState* st = &v.rs[r];
  double ke = 0.0;
  if (kPost) ke = post_slot_vm<true, kKinetic>(v, p, st, i, owner, vm_kick, fx, fy, fz);
  if (kObs) {
    const float e = ae.total(), w = aw.total();
    block_add_lane<kBlock>(owner, 0.5 * (double)e, st, kAccPair);
    block_add_lane<kBlock>(owner, 0.5 * (double)w, st, kAccVirial);
  }
  if (kPost) post_partial<kKinetic>(v, st, r, owner, ke);
}

// LJ pair forces of a staged context: block g handles the 128 particles of
// cell-order rows [128 g, 128 g + 128) (kTpa threads each).  Its first warp
// derives the group's stage layout (stage_layout, the same function the list
// build used), the block copies the stage -- pos[cell_atoms[q]] for every q
// of every window, one window per warp at a time -- into shared memory, and
// every neighbour position of the pair loop is then a shared-memory load
// instead of an L1/L2 gather.  A group whose layout fell back to slot
// entries reads global positions, as k_lj does.  The arithmetic, the list
// order and the canonical summation order are k_lj's, so the forces, energies
// and virial are bit-identical to k_lj's for the same list.
template <bool kObs, int kMode, int kTpa, int kUnroll, bool kNoL1, int kNt>
__global__ void __launch_bounds__(kBlock* kTpa) k_lj_staged(DeviceView v) {
  constexpr int kThreads = kBlock * kTpa;
  constexpr bool kClamp = kMode == kForceClamp;
  constexpr bool kPost = kMode >= kForcePost;
  constexpr bool kKinetic = kMode == kForcePostKinetic || (kPost && kObs);
  extern __shared__ float4 stage[];  // v.stage_cap + 1 entries
  __shared__ StageLayout lay;
  __shared__ LjCoeff table[kMaxTypes * kMaxTypes];
  const uint32_t g = blockIdx.x;
  const uint32_t r = v.block_replica[g];
  const ReplicaParams& p = v.rp[r];
  const int nt = p.n_types;
  for (int t = threadIdx.x; t < nt * nt; t += kThreads) table[t] = v.lj[p.lj_offset + t];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  if (warp == 0) stage_layout(v, p, g, lane, v.stage_cap, lay);
  __syncthreads();
  const bool staged = lay.n_win != 0u;
  if (staged) {
    const uint32_t n_win = lay.n_win;
    for (uint32_t w = warp; w < n_win; w += kThreads / 32) {
      const uint32_t q0 = lay.qbeg[w], b = lay.base[w];
      const uint32_t len = (w + 1u < n_win ? lay.base[w + 1u] : lay.size) - b;
      for (uint32_t t = lane; t < len; t += 32u) stage[b + t] = v.pos[v.cell_atoms[q0 + t]];
    }
    if (threadIdx.x == 0) stage[lay.size] = v.pos[v.n_slots];  // the far particle
    __syncthreads();
  }

  const uint32_t sub = threadIdx.x % kTpa;
  const uint32_t q = g * kBlock + threadIdx.x / kTpa;
  const bool real = q >= lay.q_first && q < lay.q_end;
  // Padding rows are padding slots (inert, never written).
  const uint32_t i = real ? v.cell_atoms[q] : q;
  LjAcc<kTpa> ax, ay, az, ae, aw;
  float4 vm_kick = make_float4(0.f, 0.f, 0.f, 1.f);
  ax.zero();
  ay.zero();
  az.zero();
  ae.zero();
  aw.zero();
  {
    const float4 xi = v.pos[i];
    if (kPost) vm_kick = (real && sub == 0u) ? v.vel[i] : make_float4(0.f, 0.f, 0.f, 1.f);
    CoeffRow<kNt> coeff;
    coeff.init(table + __float_as_int(xi.w) * nt);
    const uint32_t n = real ? v.nbr_count[q] : 0u;
    const uint32_t n_warp = __reduce_max_sync(kFull, n);
    const float rc2 = p.force_cut_sq;
    const float hmin = fminf(p.half[0], fminf(p.half[1], p.half[2]));
    const float half_min_sq = hmin * hmin;
    const float rcm = 1.001f * sqrtf(rc2) + 1e-6f * fmaxf(p.len[0], fmaxf(p.len[1], p.len[2]));
    const bool inside = !real ||
        (xi.x - p.lo[0] >= rcm && p.lo[0] + p.len[0] - xi.x > rcm &&
         xi.y - p.lo[1] >= rcm && p.lo[1] + p.len[1] - xi.y > rcm &&
         xi.z - p.lo[2] >= rcm && p.lo[2] + p.len[2] - xi.z > rcm);
    const bool all_inside = __all_sync(kFull, inside);
    if (staged) {
      if (all_inside) {
        lj_pairs<kObs, kClamp, kTpa, kUnroll, kNoL1, false, kNt, true>(
            v, p, coeff, xi, q, stage, lay.size, sub, n, n_warp, rc2, half_min_sq, ax, ay, az,
            ae, aw);
      } else {
        lj_pairs<kObs, kClamp, kTpa, kUnroll, kNoL1, true, kNt, true>(
            v, p, coeff, xi, q, stage, lay.size, sub, n, n_warp, rc2, half_min_sq, ax, ay, az,
            ae, aw);
      }
    } else {
      if (all_inside) {
        lj_pairs<kObs, kClamp, kTpa, kUnroll, kNoL1, false, kNt>(
            v, p, coeff, xi, q, v.pos, v.n_slots, sub, n, n_warp, rc2, half_min_sq, ax, ay, az,
            ae, aw);
      } else {
        lj_pairs<kObs, kClamp, kTpa, kUnroll, kNoL1, true, kNt>(
            v, p, coeff, xi, q, v.pos, v.n_slots, sub, n, n_warp, rc2, half_min_sq, ax, ay, az,
            ae, aw);
      }
    }
  }
  const float fx = ax.total(), fy = ay.total(), fz = az.total();
  const bool owner = real && sub == 0u;
  if (owner) v.force[i] = make_float4(fx, fy, fz, 0.f);
  ReplicaState* st = &v.rs[r];
  double ke = 0.0;
  if (kPost) ke = post_slot_vm<true, kKinetic>(v, p, st, i, owner, vm_kick, fx, fy, fz);
  if (kObs) {
    const float e = ae.total(), w = aw.total();
    block_add_lane<kThreads>(owner, 0.5 * (double)e, st, kAccPair);
    block_add_lane<kThreads>(owner, 0.5 * (double)w, st, kAccVirial);
  }
  if (kPost) post_partial<kKinetic>(v, st, r, owner, ke);
}

// Slot-indexed copy of a staged context's list (debug views): out_count[slot]
// and out[slot * cap + k] = neighbour slot, decoding stage indices through the
// group's layout.  One block of 128 threads per group.
__global__ void __launch_bounds__(kBlock) k_list_to_slots(DeviceView v, uint32_t cap,
                                                          uint32_t* out_count, uint32_t* out) {
  __shared__ StageLayout lay;
  const uint32_t g = blockIdx.x;
  const ReplicaParams& p = v.rp[v.block_replica[g]];
  if (threadIdx.x < 32) stage_layout(v, p, g, threadIdx.x, v.stage_cap, lay);
  __syncthreads();
  const uint32_t q = g * kBlock + threadIdx.x;
  if (q < lay.q_first || q >= lay.q_end) return;
  const uint32_t i = v.cell_atoms[q];
  const uint32_t n = v.nbr_count[q];
  out_count[i] = n;
  const uint32_t* list = v.nbr + nbr_index(q, 0, v.nbr_stride);
  for (uint32_t k = 0; k < n && k < cap; ++k) {
    uint32_t e = list[(size_t)k * kGroup];
    if (lay.n_win != 0u) {
      uint32_t w = 0;  // last window whose base <= e
      while (w + 1u < lay.n_win && lay.base[w + 1u] <= e) ++w;
      e = v.cell_atoms[lay.qbeg[w] + (e - lay.base[w])];
    }
    out[(size_t)i * cap + k] = e;
  }
}

// ---------------------------------------------------------------------------
// Bonded terms, gathered per particle.
struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ float dot3(V3 a, V3 b) {
  return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, __fmul_rn(a.x, b.x)));
}
__device__ __forceinline__ V3 cross3(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ V3 axpy(float a, V3 x, V3 y) {
  return v3(__fmaf_rn(a, x.x, y.x), __fmaf_rn(a, x.y, y.y), __fmaf_rn(a, x.z, y.z));
}
__device__ __forceinline__ V3 scal(float a, V3 x) { return v3(a * x.x, a * x.y, a * x.z); }

__device__ __forceinline__ V3 arm(const DeviceView& v, const ReplicaParams& p,
                                  uint32_t tag_a, uint32_t tag_b) {
  const float4 a = v.pos[v.slot_of_tag[tag_a]];
  const float4 b = v.pos[v.slot_of_tag[tag_b]];
  return v3(acc_delta(a.x, b.x, p.len[0], p.half[0]),
            acc_delta(a.y, b.y, p.len[1], p.half[1]),
            acc_delta(a.z, b.z, p.len[2], p.half[2]));
}

// |d| and |d| - r0 of a float vector d, the stretch accurate to a few units
// of 2^-48 relative to |d| instead of 2^-24: the squares are split into
// rounded products and their exact errors (fma), the two additions into sums
// and their exact errors (TwoSum), and one Newton step corrects the float
// square root against the compensated sum.  A stiff bond (k = 500 at r0 =
// 0.97) turns the 2^-24 error of a plain r - r0 into a force error of
// ~3e-5, near the 1e-5 relative-RMS force bar of a relaxed melt, whose total
// forces are small next to the bonded ones they cancel.
__device__ __forceinline__ float two_sum_err(float a, float b, float s) {
  const float bb = __fsub_rn(s, a);
  return __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}
__device__ __forceinline__ float bond_length(V3 d, float r0, float& stretch) {
  const float px = __fmul_rn(d.x, d.x), py = __fmul_rn(d.y, d.y), pz = __fmul_rn(d.z, d.z);
  const float ex = __fmaf_rn(d.x, d.x, -px), ey = __fmaf_rn(d.y, d.y, -py),
              ez = __fmaf_rn(d.z, d.z, -pz);
  const float s1 = __fadd_rn(px, py);
  const float t1 = two_sum_err(px, py, s1);
  const float q = __fadd_rn(s1, pz);
  const float t2 = two_sum_err(s1, pz, q);
  const float lo = __fadd_rn(__fadd_rn(__fadd_rn(ex, ey), __fadd_rn(ez, t1)), t2);
  const float r = sqrtf(q);
  if (r == 0.0f) {
    stretch = -r0;
    return 0.0f;
  }
  // sqrt(q + lo) = r + (q - r^2 + lo) / (2 r) to second order; q - r^2 is
  // exact in one fma.
  const float corr = __fdiv_rn(__fadd_rn(__fmaf_rn(-r, r, q), lo), __fmul_rn(2.0f, r));
  stretch = __fadd_rn(__fsub_rn(r, r0), corr);
  return __fadd_rn(r, corr);
}

// Force on member `role` of a harmonic bond; energy and virial of the whole
// term.  U = 0.5 k (r - r0)^2.
__device__ void bond_forces(const DeviceView& v, const ReplicaParams& p, uint32_t idx,
                            V3 (&f)[4], float& energy, float& virial) {
  const uint4 t = v.bonds[idx];
  const BondCoeff c = v.bond_coeff[t.z];
  const V3 d = arm(v, p, t.x, t.y);
  float s;
  const float r = bond_length(d, c.r0, s);
  energy = 0.5f * c.k * s * s;
  if (r == 0.0f) {
    virial = 0.f;
    f[0] = f[1] = v3(0.f, 0.f, 0.f);
    return;
  }
  const float sc = -c.k * s / r;
  virial = -c.k * s * r;
  f[0] = scal(sc, d);
  f[1] = scal(-sc, d);
}

// U = 0.5 k (theta - theta0)^2 with the reference's conventions: sin(theta)
// floored at 1e-3 where sin^2 <= 1e-6, theta = 0 (energy only) on a
// zero-length arm.  Written for float accuracy near straight angles, where
// the reference's form (cos clamped to [-1, 1], theta = acos(cos), sin =
// sqrt(1 - cos^2)) loses digits to cancellation: sin(theta) comes from the
// cross product n = a1 x a2 (|n| = r1 r2 sin), theta = atan2(|n|, a1.a2),
// and the force on i, a (cos a1 / r1^2 - a2 / (r1 r2)) with a = -k dtheta /
// sin, is evaluated as a (a1 x n) / (r1^2 r1 r2) = -k dtheta (a1 x n) /
// (r1^2 |n|) (likewise for k); the same quantities in exact arithmetic.
__device__ void angle_forces(const DeviceView& v, const ReplicaParams& p, uint32_t idx,
                             V3 (&f)[4], float& energy, float& virial) {
  const uint4 t = v.angles[idx];
  const AngleCoeff c = v.angle_coeff[t.w];
  const V3 a1 = arm(v, p, t.x, t.y);   // i - j
  const V3 a2 = arm(v, p, t.z, t.y);   // k - j
  const float q1 = dot3(a1, a1);
  const float q2 = dot3(a2, a2);
  if (q1 == 0.0f || q2 == 0.0f) {
    energy = 0.5f * c.k * c.theta0 * c.theta0;
    virial = 0.f;
    f[0] = f[1] = f[2] = v3(0.f, 0.f, 0.f);
    return;
  }
  const V3 n = cross3(a1, a2);
  const float qn = dot3(n, n);
  const float nm = sqrtf(qn);
  const float dt = dot3(a1, a2);
  const float theta = atan2f(nm, dt);
  const float dth = theta - c.theta0;
  energy = 0.5f * c.k * dth * dth;
  V3 fi, fk;
  if (qn <= 1.0e-6f * q1 * q2) {
    // The reference's floor: sin = 1e-3.
    const float r1 = sqrtf(q1), r2 = sqrtf(q2);
    const float cs = fminf(1.0f, fmaxf(-1.0f, dt / (r1 * r2)));
    const float a = -c.k * dth * 1.0e3f;
    const float c11 = a * cs / q1;
    const float c12 = -a / (r1 * r2);
    const float c22 = a * cs / q2;
    fi = axpy(c12, a2, scal(c11, a1));
    fk = axpy(c12, a1, scal(c22, a2));
  } else {
    const float g = -c.k * dth / nm;
    fi = scal(g / q1, cross3(a1, n));
    fk = scal(g / q2, cross3(n, a2));
  }
  virial = dot3(a1, fi) + dot3(a2, fk);
  f[0] = fi;
  f[1] = v3(-(fi.x + fk.x), -(fi.y + fk.y), -(fi.z + fk.z));
  f[2] = fk;
}

// U = k (1 + d cos(n phi)), signed phi; singular geometry contributes energy
// only (k(1+d) if n == 0, else k).  phi = atan2(|b1| b0.(b1 x b2),
// (b0 x b1).(b1 x b2)): the reference's acos of the normalised cosine with
// the sign of b0.(b1 x b2), in a form that keeps float accuracy near
// phi = 0 and pi (cis and trans), where acos loses digits.
__device__ void dihedral_forces(const DeviceView& v, const ReplicaParams& p, uint32_t idx,
                                V3 (&f)[4], float& energy, float& virial) {
  const uint4 t = v.dihedrals[idx];
  const DihedralCoeff c = v.dihedral_coeff[v.dihedral_type[idx]];
  const V3 b0 = arm(v, p, t.x, t.y);   // i - j
  const V3 b1 = arm(v, p, t.z, t.y);   // k - j
  const V3 b2 = arm(v, p, t.z, t.w);   // k - l
  const V3 m = cross3(b0, b1);
  const V3 n = cross3(b1, b2);
  const float q1 = dot3(b1, b1);
  const float qm = dot3(m, m);
  const float qn = dot3(n, n);
  if (q1 == 0.0f || qm == 0.0f || qn == 0.0f) {
    energy = c.n == 0 ? c.k * (1.0f + (float)c.d) : c.k;
    virial = 0.f;
    f[0] = f[1] = f[2] = f[3] = v3(0.f, 0.f, 0.f);
    return;
  }
  const float l1 = sqrtf(q1);
  const float phi = atan2f(l1 * dot3(b0, n), dot3(m, n));
  const float arg = (float)c.n * phi;
  float sn, cn;
  sincosf(arg, &sn, &cn);
  energy = c.k * (1.0f + (float)c.d * cn);
  const float de = -c.k * (float)c.d * (float)c.n * sn;
  const V3 fi = scal(-de * l1 / qm, m);
  const V3 fl = scal(de * l1 / qn, n);
  const float inv_q1 = 1.0f / q1;
  const V3 s = v3(fi.x * (dot3(b0, b1) * inv_q1) - fl.x * (dot3(b2, b1) * inv_q1),
                  fi.y * (dot3(b0, b1) * inv_q1) - fl.y * (dot3(b2, b1) * inv_q1),
                  fi.z * (dot3(b0, b1) * inv_q1) - fl.z * (dot3(b2, b1) * inv_q1));
  const V3 fj = v3(s.x - fi.x, s.y - fi.y, s.z - fi.z);
  const V3 fk = v3(-(s.x + fl.x), -(s.y + fl.y), -(s.z + fl.z));
  const V3 lj = v3(b1.x - b2.x, b1.y - b2.y, b1.z - b2.z);
  virial = dot3(b0, fi) + dot3(b1, fk) + dot3(lj, fl);
  f[0] = fi;
  f[1] = fj;
  f[2] = fk;
  f[3] = fl;
}

// Bonded terms, one thread per term (bonds, then angles, then dihedrals in
// one index space): the term is evaluated once and the force on each member
// goes to that member's membership entry (term_mem), with the term's energy
// in the first member's entry (.w) and, for observables, its virial
// beside it.  k_bonded then sums each particle's entries in membership
// order, so the sum order is fixed and no force atomics exist.
template <bool kObs>
__global__ void __launch_bounds__(kBlock) k_bonded_terms(DeviceView v) {
  const uint32_t t = blockIdx.x * kBlock + threadIdx.x;
  const uint32_t nb = v.n_bond_terms, na = v.n_angle_terms, nd = v.n_dihedral_terms;
  if (t >= nb + na + nd) return;
  uint32_t kind, idx, first_tag, nm, mem;
  if (t < nb) {
    kind = kTermBond, idx = t, first_tag = v.bonds[idx].x, nm = 2u, mem = 2u * idx;
  } else if (t < nb + na) {
    kind = kTermAngle, idx = t - nb, first_tag = v.angles[idx].x, nm = 3u;
    mem = 2u * nb + 3u * idx;
  } else {
    kind = kTermDihedral, idx = t - nb - na, first_tag = v.dihedrals[idx].x, nm = 4u;
    mem = 2u * nb + 3u * na + 4u * idx;
  }
  const ReplicaParams& p = v.rp[v.block_replica[v.slot_of_tag[first_tag] / (uint32_t)kBlock]];
  V3 f[4];
  float en = 0.f, vir = 0.f;
  if (kind == kTermBond) {
    bond_forces(v, p, idx, f, en, vir);
  } else if (kind == kTermAngle) {
    angle_forces(v, p, idx, f, en, vir);
  } else {
    dihedral_forces(v, p, idx, f, en, vir);
  }
  for (uint32_t m = 0; m < nm; ++m) {
    const uint32_t e = v.term_mem[mem + m];
    v.bonded_contrib[e] = make_float4(f[m].x, f[m].y, f[m].z, m == 0u ? en : 0.f);
    if (kObs && m == 0u) v.bonded_vir[e] = vir;
  }
}

// Per particle: the bonded force from its membership entries (in membership
// order) added to the pair force, then (post modes) the second half-kick.
template <bool kObs, int kMode>
__global__ void __launch_bounds__(kBlock) k_bonded(DeviceView v) {
  constexpr bool kPost = kMode >= kForcePost;
  constexpr bool kKinetic = kMode == kForcePostKinetic || (kPost && kObs);
  const uint32_t b = blockIdx.x;
  const uint32_t r = v.block_replica[b];
  const ReplicaParams& p = v.rp[r];
  const uint32_t i = b * kBlock + threadIdx.x;
  const bool real = (i - p.atom_begin) < p.n_atoms;
  float eb = 0.f, ea = 0.f, ed = 0.f, w = 0.f;
  float4 fo = make_float4(0.f, 0.f, 0.f, 0.f);
  if (real) {
    const uint32_t t = v.tag[i];
    const uint32_t e0 = v.term_off[t];
    const uint32_t e1 = v.term_off[t + 1];
    if (e1 > e0) {
      V3 f = v3(0.f, 0.f, 0.f);
      for (uint32_t e = e0; e < e1; ++e) {
        const float4 c = v.bonded_contrib[e];
        f.x = __fadd_rn(f.x, c.x);
        f.y = __fadd_rn(f.y, c.y);
        f.z = __fadd_rn(f.z, c.z);
        if (kObs) {
          const uint32_t m = v.term[e];
          if (((m >> 28) & 3u) == 0u) {
            const uint32_t kind = m >> 30;
            if (kind == kTermBond) eb += c.w;
            else if (kind == kTermAngle) ea += c.w;
            else ed += c.w;
            w += v.bonded_vir[e];
          }
        }
      }
      fo = v.force[i];
      fo.x = __fadd_rn(fo.x, f.x);
      fo.y = __fadd_rn(fo.y, f.y);
      fo.z = __fadd_rn(fo.z, f.z);
      v.force[i] = fo;
    } else if (kPost) {
      fo = v.force[i];
    }
  }
  ReplicaState* st = &v.rs[r];
  double ke = 0.0;
  if (kPost) ke = post_slot<true, kKinetic>(v, p, st, i, real, fo.x, fo.y, fo.z);
  if (kObs) {
    block_add_lane<kBlock>(real, eb, st, kAccBond);
    block_add_lane<kBlock>(real, ea, st, kAccAngle);
    block_add_lane<kBlock>(real, ed, st, kAccDihedral);
    block_add_lane<kBlock>(real, w, st, kAccVirial);
  }
  if (kPost) post_partial<kKinetic>(v, st, r, real, ke);
}

// ---------------------------------------------------------------------------
// post: second half-kick and kinetic energy (FP64 per slot, one fixed-point
// bucket add per block); k_post_finish then does the per-replica epilogue
// (observables, Berendsen lambda for the next step, applied lazily by pre,
// step counter).  The same per-slot work runs inside the last force kernel
// when the schedule fuses the kick.

template <bool kKick, bool kObs, bool kKinetic>
__global__ void __launch_bounds__(kBlock) k_post(DeviceView v) {
  wait_prior_grid();
  const uint32_t b = blockIdx.x;
  const uint32_t r = v.block_replica[b];
  const ReplicaParams& p = v.rp[r];
  ReplicaState* st = &v.rs[r];
  const uint32_t i = b * kBlock + threadIdx.x;
  const bool real = (i - p.atom_begin) < p.n_atoms;
  float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
  if (kKick && real) f = v.force[i];
  const double ke = post_slot<kKick, kKinetic || kObs>(v, p, st, i, real, f.x, f.y, f.z);
  post_partial_block<kKinetic || kObs>(v, st, r, real, ke);
}

// Applies the pending Berendsen scale so host reads see the scaled velocities.
__global__ void k_apply_lambda(DeviceView v) {
  const uint32_t b = blockIdx.x;
  const uint32_t r = v.block_replica[b];
  const ReplicaParams& p = v.rp[r];
  ReplicaState* st = &v.rs[r];
  const uint32_t i = b * kBlock + threadIdx.x;
  const float lam = (float)st->lambda;
  if ((i - p.atom_begin) < p.n_atoms && lam != 1.0f) {
    float4 u = v.vel[i];
    u.x = __fmul_rn(u.x, lam);
    u.y = __fmul_rn(u.y, lam);
    u.z = __fmul_rn(u.z, lam);
    v.vel[i] = u;
  }
  if (arrive_last(&st->done_pre, p.n_pad / kBlock) && threadIdx.x == 0) {
    st->lambda = 1.0;
    st->done_pre = 0u;
  }
}

__global__ void k_scatter_state(DeviceView v, const float* pos_tag,
                                const float* vel_tag, uint32_t n_tags) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tags) return;
  const uint32_t s = v.slot_of_tag[t];
  if (pos_tag) {
    float4 x = v.pos[s];
    x.x = pos_tag[3 * (size_t)t];
    x.y = pos_tag[3 * (size_t)t + 1];
    x.z = pos_tag[3 * (size_t)t + 2];
    v.pos[s] = x;
  }
  if (vel_tag) {
    float4 u = v.vel[s];
    u.x = vel_tag[3 * (size_t)t];
    u.y = vel_tag[3 * (size_t)t + 1];
    u.z = vel_tag[3 * (size_t)t + 2];
    v.vel[s] = u;
  }
}

__global__ void k_gather_state(DeviceView v, float* pos_tag, float* vel_tag,
                               uint32_t n_tags) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tags) return;
  const uint32_t s = v.slot_of_tag[t];
  if (pos_tag) {
    const float4 x = v.pos[s];
    pos_tag[3 * (size_t)t] = x.x;
    pos_tag[3 * (size_t)t + 1] = x.y;
    pos_tag[3 * (size_t)t + 2] = x.z;
  }
  if (vel_tag) {
    const float4 u = v.vel[s];
    vel_tag[3 * (size_t)t] = u.x;
    vel_tag[3 * (size_t)t + 1] = u.y;
    vel_tag[3 * (size_t)t + 2] = u.z;
  }
}

void check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    throw std::runtime_error(std::string("CUDA launch of ") + what +
                             " failed: " + cudaGetErrorString(e));
  }
}

// Launches a kernel as a programmatic dependent of the previous work in the
// stream (also inside a stream capture): its blocks may be scheduled while
// that work drains, hiding the launch gap, and wait in wait_prior_grid()
// before touching its results.  Used for the short per-step kernels that
// follow another kernel directly.
template <typename... P, typename... A>
void launch_dependent(void (*kernel)(P...), dim3 grid, dim3 block, cudaStream_t stream,
                      const char* what, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
  if (e != cudaSuccess) {
    throw std::runtime_error(std::string("CUDA launch of ") + what +
                             " failed: " + cudaGetErrorString(e));
  }
}

}  // namespace

void launch_pre(const StepLaunch& l, int mode, cudaGraphConditionalHandle cond, bool use_cond) {
  const uint32_t dg = (l.v.n_replicas + 127) / 128;
  if (mode == kPreDescent) {
    launch_dependent(k_pre<kPreDescent>, dim3(l.v.n_blocks), dim3(kBlock), l.stream, "pre", l.v,
                     l.sd_dmax, l.sd_fref);
    launch_dependent(k_decide<kPreDescent>, dim3(dg), dim3(128), l.stream, "decide", l.v, cond,
                     use_cond ? 1 : 0);
  } else {
    launch_dependent(k_pre<kPreVerlet>, dim3(l.v.n_blocks), dim3(kBlock), l.stream, "pre", l.v,
                     0.f, 0.f);
    launch_dependent(k_decide<kPreVerlet>, dim3(dg), dim3(128), l.stream, "decide", l.v, cond,
                     use_cond ? 1 : 0);
  }
  check_launch("decide");
}

void launch_project_exclusions(const StepLaunch& l, bool force_all) {
  if (l.excl_cap == 0) return;
  k_project_exclusions<<<l.v.n_blocks, kBlock, 0, l.stream>>>(l.v, force_all ? 1 : 0);
  check_launch("project_exclusions");
}

void launch_rebuild(const StepLaunch& l, bool force_all, bool count_build) {
  if (force_all) {
    k_force_rebuild_flags<<<(l.v.n_replicas + 127) / 128, 128, 0, l.stream>>>(
        l.v, count_build ? 1 : 0);
    check_launch("force_rebuild_flags");
  }
  // With the block list, the per-slot kernels of the chain walk the
  // rebuilding replicas' blocks with a grid of chain_grid blocks.
  const uint32_t sg = l.v.chain_block_list ? l.chain_grid : l.v.n_blocks;
  if (l.v.chain_block_list) {
    k_chain_blocks<<<1, kScanThreads, 0, l.stream>>>(l.v);
    check_launch("chain blocks");
  }
  k_bin<<<sg, kBlock, 0, l.stream>>>(l.v);
  check_launch("bin");
  if (l.v.n_scan_chunks == l.v.n_replicas) {  // every replica fits one chunk
    k_scan_single<<<l.v.n_replicas, kScanThreads, 0, l.stream>>>(l.v);
    check_launch("scan");
  } else {
    k_scan_sum<<<l.v.n_scan_chunks, kScanThreads, 0, l.stream>>>(l.v);
    check_launch("scan sum");
    k_scan<<<l.v.n_replicas, kScanThreads, 0, l.stream>>>(l.v);
    check_launch("scan");
    k_scan_cells<<<l.v.n_scan_chunks, kScanThreads, 0, l.stream>>>(l.v);
    check_launch("scan cells");
  }
  k_scatter<<<sg, kBlock, 0, l.stream>>>(l.v);
  check_launch("scatter");
  if (l.any_sparse) {
    k_cellsort_sparse<<<(l.v.total_cells + kBlock - 1) / kBlock, kBlock, 0, l.stream>>>(l.v);
    check_launch("cellsort sparse");
  }
  k_cellsort<<<(l.v.total_cells + kBlock / 32 - 1) / (kBlock / 32), kBlock, 0, l.stream>>>(l.v);
  check_launch("cellsort");
  k_reorder_gather<<<sg, kBlock, 0, l.stream>>>(l.v);
  check_launch("reorder_gather");
  k_reorder_commit<<<sg, kBlock, 0, l.stream>>>(l.v);
  check_launch("reorder_commit");
  if (l.excl_cap > 0) {
    k_project_exclusions<<<l.v.n_blocks, kBlock, 0, l.stream>>>(l.v, 0);
    check_launch("project_exclusions");
  }
  const uint32_t bg = (l.v.total_cells + kBuildWarps - 1) / kBuildWarps;
#define BB_BUILD_Q(cap, q)                                                             \
  do {                                                                                  \
    if (l.any_dense) k_build<cap, q><<<bg, kBlock, 0, l.stream>>>(l.v);                 \
    if (l.any_sparse) k_build_sparse<cap, q><<<l.v.n_blocks, kBlock, 0, l.stream>>>(l.v); \
  } while (0)
#define BB_BUILD(cap)           \
  do {                          \
    if (l.v.list_by_q) {        \
      BB_BUILD_Q(cap, true);    \
    } else {                    \
      BB_BUILD_Q(cap, false);   \
    }                           \
  } while (0)
  switch (l.excl_cap) {
    case 0: BB_BUILD(0); break;
    case 4: BB_BUILD(4); break;
    case 8: BB_BUILD(8); break;
    case 16: BB_BUILD(16); break;
    case 32: BB_BUILD(32); break;
    case 64: BB_BUILD(64); break;
    default: throw std::runtime_error("unsupported exclusion capacity");
  }
#undef BB_BUILD
#undef BB_BUILD_Q
  check_launch("build");
}

// Steps that need observables (thermo rows, eval) use the general-table
// kernel at depth 4 with the tuned threads per particle; every variant sums
// forces in the same order, so the choice never shows in the results.
template <int kTpa>
void launch_lj_obs(const StepLaunch& l, int mode) {
  const dim3 grid(l.v.n_blocks * kTpa);
  if (mode == kForcePlain) {
    k_lj<true, kForcePlain, kTpa, 4, true, 0><<<grid, kBlock, 0, l.stream>>>(l.v);
  } else {  // the kinetic total is part of the observables
    k_lj<true, kForcePost, kTpa, 4, true, 0><<<grid, kBlock, 0, l.stream>>>(l.v);
  }
}

template <int kTpa, int kUnroll, bool kNoL1, int kNt>
void launch_lj_tpa(const StepLaunch& l, int mode) {
  const dim3 grid(l.v.n_blocks * kTpa);
#define BB_LJ(m) k_lj<false, m, kTpa, kUnroll, kNoL1, kNt><<<grid, kBlock, 0, l.stream>>>(l.v)
  switch (mode) {
    case kForcePlain: BB_LJ(kForcePlain); break;
    case kForcePost: BB_LJ(kForcePost); break;
    default: BB_LJ(kForcePostKinetic); break;
  }
#undef BB_LJ
}

template <int kTpa, int kUnroll, bool kNoL1>
void launch_lj_nt(const StepLaunch& l, int mode) {
  switch (l.lj_types) {
    case 1: launch_lj_tpa<kTpa, kUnroll, kNoL1, 1>(l, mode); break;
    case 2: launch_lj_tpa<kTpa, kUnroll, kNoL1, 2>(l, mode); break;
    default: launch_lj_tpa<kTpa, kUnroll, kNoL1, 0>(l, mode); break;
  }
}

namespace {

// Staged contexts: every pair-force launch goes to k_lj_staged (the list
// rows are cell-order rows there), with (stage_cap + 1) float4 of dynamic
// shared memory.
size_t staged_smem(const StepLaunch& l) { return (size_t)(l.v.stage_cap + 1u) * sizeof(float4); }

template <bool kObs, int kMode, int kTpa, int kUnroll, int kNt>
void staged_one(const StepLaunch& l) {
  k_lj_staged<kObs, kMode, kTpa, kUnroll, true, kNt>
      <<<l.v.n_blocks, kBlock * kTpa, staged_smem(l), l.stream>>>(l.v);
}

template <bool kObs, int kMode, int kTpa, int kUnroll, int kNt>
void staged_attr(size_t smem) {
  const cudaError_t e =
      cudaFuncSetAttribute(k_lj_staged<kObs, kMode, kTpa, kUnroll, true, kNt>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    throw std::runtime_error(std::string("staged pair kernel shared memory: ") +
                             cudaGetErrorString(e));
  }
}

template <int kTpa, int kUnroll, int kNt>
void staged_attr_modes(size_t smem) {
  staged_attr<false, kForcePlain, kTpa, kUnroll, kNt>(smem);
  staged_attr<false, kForcePost, kTpa, kUnroll, kNt>(smem);
  staged_attr<false, kForcePostKinetic, kTpa, kUnroll, kNt>(smem);
}

template <int kTpa, int kUnroll, int kNt>
void staged_plain(const StepLaunch& l, int mode) {
  switch (mode) {
    case kForcePlain: staged_one<false, kForcePlain, kTpa, kUnroll, kNt>(l); break;
    case kForcePost: staged_one<false, kForcePost, kTpa, kUnroll, kNt>(l); break;
    default: staged_one<false, kForcePostKinetic, kTpa, kUnroll, kNt>(l); break;
  }
}

template <int kTpa, int kUnroll>
void staged_plain_nt(const StepLaunch& l, int mode) {
  switch (l.lj_types) {
    case 1: staged_plain<kTpa, kUnroll, 1>(l, mode); break;
    case 2: staged_plain<kTpa, kUnroll, 2>(l, mode); break;
    default: staged_plain<kTpa, kUnroll, 0>(l, mode); break;
  }
}

void launch_forces_staged(const StepLaunch& l, bool observables, bool clamp, int mode) {
  if (clamp) {
    staged_one<false, kForceClamp, 2, 4, 0>(l);
  } else if (observables) {
    const bool plain = mode == kForcePlain;
    switch (l.lj_tpa) {
      case 2:
        plain ? staged_one<true, kForcePlain, 2, 4, 0>(l) : staged_one<true, kForcePost, 2, 4, 0>(l);
        break;
      case 4:
        plain ? staged_one<true, kForcePlain, 4, 4, 0>(l) : staged_one<true, kForcePost, 4, 4, 0>(l);
        break;
      default:
        plain ? staged_one<true, kForcePlain, 1, 4, 0>(l) : staged_one<true, kForcePost, 1, 4, 0>(l);
        break;
    }
  } else {
    const int key = l.lj_tpa * 10 + l.lj_unroll;
    switch (key) {
      case 14: staged_plain_nt<1, 4>(l, mode); break;
      case 18: staged_plain_nt<1, 8>(l, mode); break;
      case 24: staged_plain_nt<2, 4>(l, mode); break;
      case 28: staged_plain_nt<2, 8>(l, mode); break;
      case 44: staged_plain_nt<4, 4>(l, mode); break;
      case 48: staged_plain_nt<4, 8>(l, mode); break;
      default: throw std::runtime_error("unsupported staged pair-force schedule");
    }
  }
  check_launch("lj_staged");
}

}  // namespace

// Raises the dynamic shared-memory limit of every staged pair-force variant to
// `smem` bytes (once per context, outside any stream capture).
void prepare_staged_kernels(size_t smem) {
  staged_attr<false, kForceClamp, 2, 4, 0>(smem);
  staged_attr<true, kForcePlain, 1, 4, 0>(smem);
  staged_attr<true, kForcePost, 1, 4, 0>(smem);
  staged_attr<true, kForcePlain, 2, 4, 0>(smem);
  staged_attr<true, kForcePost, 2, 4, 0>(smem);
  staged_attr<true, kForcePlain, 4, 4, 0>(smem);
  staged_attr<true, kForcePost, 4, 4, 0>(smem);
#define BB_ATTR(t, u)                    \
  staged_attr_modes<t, u, 0>(smem);      \
  staged_attr_modes<t, u, 1>(smem);      \
  staged_attr_modes<t, u, 2>(smem);
  BB_ATTR(1, 4) BB_ATTR(1, 8) BB_ATTR(2, 4) BB_ATTR(2, 8) BB_ATTR(4, 4) BB_ATTR(4, 8)
#undef BB_ATTR
}

void launch_list_to_slots(const StepLaunch& l, uint32_t cap, uint32_t* out_count, uint32_t* out) {
  k_list_to_slots<<<l.v.n_blocks, kBlock, 0, l.stream>>>(l.v, cap, out_count, out);
  check_launch("list_to_slots");
}

void launch_forces(const StepLaunch& l, bool observables, bool clamp, bool post, int parts) {
  const bool fuse = post && l.fuse_post != 0;
  const int fin = !fuse ? kForcePlain : (l.need_kinetic ? kForcePostKinetic : kForcePost);
  const bool bonded = l.v.has_bonded != 0 && (parts & kForceBonded) != 0;
  if ((parts & kForcePair) == 0) {
    // bonded terms alone (profiling)
  } else if (l.v.list_by_q) {
    launch_forces_staged(l, observables, clamp, bonded ? kForcePlain : fin);
  } else if (clamp) {
    k_lj<false, kForceClamp, 1, 8, false, 0><<<l.v.n_blocks, kBlock, 0, l.stream>>>(l.v);
  } else if (observables) {
    const int mode = bonded ? kForcePlain : fin;
    switch (l.lj_tpa) {
      case 2: launch_lj_obs<2>(l, mode); break;
      case 4: launch_lj_obs<4>(l, mode); break;
      default: launch_lj_obs<1>(l, mode); break;
    }
  } else {
    const int mode = bonded ? kForcePlain : fin;
    // (threads per particle, batch depth, list load policy) -> one instantiation
    const int key = l.lj_tpa * 100 + l.lj_unroll * 10 + (l.lj_no_l1 ? 1 : 0);
    switch (key) {
#define BB_CASE(t, u, pf) \
  case t * 100 + u * 10 + pf: launch_lj_nt<t, u, pf != 0>(l, mode); break;
      BB_CASE(1, 8, 0) BB_CASE(1, 8, 1) BB_CASE(1, 4, 0) BB_CASE(1, 4, 1)
      BB_CASE(2, 8, 0) BB_CASE(2, 8, 1) BB_CASE(2, 4, 0) BB_CASE(2, 4, 1)
      BB_CASE(4, 8, 0) BB_CASE(4, 8, 1) BB_CASE(4, 4, 0) BB_CASE(4, 4, 1)
#undef BB_CASE
      default: throw std::runtime_error("unsupported pair-force schedule");
    }
  }
  if (parts & kForcePair) check_launch("lj");
  if (bonded) {
    const uint32_t n_terms = l.v.n_bond_terms + l.v.n_angle_terms + l.v.n_dihedral_terms;
    const uint32_t tg = (n_terms + kBlock - 1) / kBlock;
    if (tg > 0) {
      if (observables) {
        k_bonded_terms<true><<<tg, kBlock, 0, l.stream>>>(l.v);
      } else {
        k_bonded_terms<false><<<tg, kBlock, 0, l.stream>>>(l.v);
      }
      check_launch("bonded terms");
    }
#define BB_BONDED(obs, mode) k_bonded<obs, mode><<<l.v.n_blocks, kBlock, 0, l.stream>>>(l.v)
    if (observables) {
      if (fin == kForcePlain) BB_BONDED(true, kForcePlain);
      else BB_BONDED(true, kForcePost);
    } else {
      switch (fin) {
        case kForcePlain: BB_BONDED(false, kForcePlain); break;
        case kForcePost: BB_BONDED(false, kForcePost); break;
        default: BB_BONDED(false, kForcePostKinetic); break;
      }
    }
#undef BB_BONDED
    check_launch("bonded");
  }
  if (fuse) {
    const bool kin = fin == kForcePostKinetic || observables;
    const dim3 fg(l.v.n_replicas), ft(kFinishThreads);
    if (observables) {
      launch_dependent(k_post_finish<true, true, true>, fg, ft, l.stream, "post finish", l.v);
    } else if (kin) {
      launch_dependent(k_post_finish<true, false, true>, fg, ft, l.stream, "post finish", l.v);
    } else {
      launch_dependent(k_post_finish<true, false, false>, fg, ft, l.stream, "post finish", l.v);
    }
    check_launch("post finish");
  }
  if (post && !fuse) launch_post(l, true, observables);
}

void launch_post(const StepLaunch& l, bool kick, bool observables) {
  const bool kin = l.need_kinetic != 0;
  const dim3 fg(l.v.n_replicas);
  if (kick) {
    if (observables) {
      launch_dependent(k_post<true, true, true>, dim3(l.v.n_blocks), dim3(kBlock), l.stream,
                       "post", l.v);
      launch_dependent(k_post_finish<true, true, true>, dim3(fg), dim3(kFinishThreads), l.stream,
                       "post finish", l.v);
    } else if (kin) {
      launch_dependent(k_post<true, false, true>, dim3(l.v.n_blocks), dim3(kBlock), l.stream,
                       "post", l.v);
      launch_dependent(k_post_finish<true, false, true>, dim3(fg), dim3(kFinishThreads), l.stream,
                       "post finish", l.v);
    } else {
      launch_dependent(k_post<true, false, false>, dim3(l.v.n_blocks), dim3(kBlock), l.stream,
                       "post", l.v);
      launch_dependent(k_post_finish<true, false, false>, dim3(fg), dim3(kFinishThreads), l.stream,
                       "post finish", l.v);
    }
  } else {
    launch_dependent(k_post<false, true, true>, dim3(l.v.n_blocks), dim3(kBlock), l.stream,
                     "post", l.v);
    launch_dependent(k_post_finish<false, true, true>, dim3(fg), dim3(kFinishThreads), l.stream,
                     "post finish", l.v);
  }
  check_launch("post");
}

void launch_apply_lambda(const StepLaunch& l) {
  k_apply_lambda<<<l.v.n_blocks, kBlock, 0, l.stream>>>(l.v);
  check_launch("apply_lambda");
}

void launch_scatter_state(const StepLaunch& l, const float* pos_tag,
                          const float* vel_tag, uint32_t n_tags_total) {
  k_scatter_state<<<(n_tags_total + 255) / 256, 256, 0, l.stream>>>(
      l.v, pos_tag, vel_tag, n_tags_total);
  check_launch("scatter_state");
}

void launch_gather_state(const StepLaunch& l, float* pos_tag, float* vel_tag,
                         uint32_t n_tags_total) {
  k_gather_state<<<(n_tags_total + 255) / 256, 256, 0, l.stream>>>(
      l.v, pos_tag, vel_tag, n_tags_total);
  check_launch("gather_state");
}

}  // namespace bb
