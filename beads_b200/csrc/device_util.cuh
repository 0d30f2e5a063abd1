// device_util.cuh -- device helpers shared by the step kernels and the
// adjoint kernels: fixed-point totals, minimum-image differences, cell
// arithmetic and the last-block pattern.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device.cuh"

namespace bb {

constexpr unsigned kFull = 0xffffffffu;

// One slot's contribution to a fixed-point total: floor(v) and the fraction
// v - floor(v) (exact in double) truncated to units of 2^-32.
struct Fixed {
  long long whole;
  long long frac;
};

__device__ __forceinline__ Fixed to_fixed(double v, unsigned* status) {
  if (!(fabs(v) < kFixLimit)) {
    atomicOr(status, kStatusFixedOverflow);
    return Fixed{0, 0};
  }
  const double w = floor(v);
  return Fixed{(long long)w, (long long)((v - w) * kFixFrac)};
}

__device__ __forceinline__ double from_fixed(long long whole, long long frac) {
  return (double)whole + (double)frac / kFixFrac;
}

// Warp + block sum of one fixed-point contribution, two atomics per block.
template <int kThreads>
__device__ __forceinline__ void block_add_fixed(Fixed f, long long* whole, long long* frac) {
  __shared__ long long partial[2][kThreads / 32];
  long long a = f.whole, c = f.frac;
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(kFull, a, o);
    c += __shfl_down_sync(kFull, c, o);
  }
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    partial[0][warp] = a;
    partial[1][warp] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long sa = 0, sc = 0;
    for (int w = 0; w < kThreads / 32; ++w) {
      sa += partial[0][w];
      sc += partial[1][w];
    }
    if (sa != 0) atomicAdd(reinterpret_cast<unsigned long long*>(whole),
                           static_cast<unsigned long long>(sa));
    if (sc != 0) atomicAdd(reinterpret_cast<unsigned long long*>(frac),
                           static_cast<unsigned long long>(sc));
  }
  __syncthreads();
}

template <int kThreads>
__device__ __forceinline__ void block_add_lane(bool real, double v, ReplicaState* st, int lane) {
  block_add_fixed<kThreads>(real ? to_fixed(v, &st->status) : Fixed{0, 0}, &st->acc[lane],
                            &st->acc_frac[lane]);
}

// Reads and clears one fixed-point total (one thread of the replica's finish block).
__device__ __forceinline__ double take_total(ReplicaState* st, int lane) {
  unsigned long long* w = reinterpret_cast<unsigned long long*>(st->acc);
  unsigned long long* f = reinterpret_cast<unsigned long long*>(st->acc_frac);
  const long long whole = (long long)atomicExch(&w[lane], 0ull);
  const long long frac = (long long)atomicExch(&f[lane], 0ull);
  return from_fixed(whole, frac);
}

// Minimum image exactly as the reference applies it to wrapped coordinates
// (box_geometry_view.cuh:50-62): one subtraction, then one shift by L.
__device__ __forceinline__ float ref_delta(float xi, float xj, float len,
                                           float half) {
  float d = __fsub_rn(xi, xj);
  if (d > half) {
    d = __fsub_rn(d, len);
  } else if (d < -half) {
    d = __fadd_rn(d, len);
  }
  return d;
}

// Minimum image rounded once from the exact difference.  When the pair spans
// the periodic boundary the reference's form rounds xi - xj at the magnitude
// of L before shifting; here the rounding error of xi - xj is recovered with
// Knuth's TwoSum and added back after the (exact, by Sterbenz) shift by L.
__device__ __forceinline__ float acc_delta(float xi, float xj, float len,
                                           float half) {
  float d = __fsub_rn(xi, xj);
  if (fabsf(d) > half) {
    const float nxj = -xj;
    const float bp = __fsub_rn(d, xi);
    const float ap = __fsub_rn(d, bp);
    const float err = __fadd_rn(__fsub_rn(xi, ap), __fsub_rn(nxj, bp));
    const float shifted = d > 0.0f ? __fsub_rn(d, len) : __fadd_rn(d, len);
    d = __fadd_rn(shifted, err);
  }
  return d;
}

// acc_delta of two pairs on one axis in packed FP32x2 arithmetic: d = xi - xj
// as already rounded, nxj = -xj.  Every lane rounds exactly as acc_delta
// does (each packed operation rounds its halves as the scalar one would); a
// lane whose pair is not `far` keeps d.
__device__ __forceinline__ float2 acc_delta2(float2 d, float2 xi, float2 nxj, float len,
                                             float half, bool far0, bool far1) {
  const float2 bp = __fadd2_rn(d, make_float2(-xi.x, -xi.y));
  const float2 ap = __fadd2_rn(d, make_float2(-bp.x, -bp.y));
  const float2 err = __fadd2_rn(__fadd2_rn(xi, make_float2(-ap.x, -ap.y)),
                                __fadd2_rn(nxj, make_float2(-bp.x, -bp.y)));
  const float2 shift = make_float2(d.x > 0.0f ? -len : len, d.y > 0.0f ? -len : len);
  const float2 img = __fadd2_rn(__fadd2_rn(d, shift), err);
  return make_float2(far0 && fabsf(d.x) > half ? img.x : d.x,
                     far1 && fabsf(d.y) > half ? img.y : d.y);
}

// Net periodic-boundary crossings of a slot since its last list build
// (img - ref_img), three signed 10-bit fields in one word, so the
// displacement check reads 4 bytes per slot instead of both image vectors.
// Bit 31 marks a field that left [-511, 511]; the check then treats the
// slot as displaced (a crossing count that large cannot occur while the
// rebuild policy holds).
constexpr uint32_t kCrossSaturated = 0x80000000u;
__device__ __forceinline__ int cross_field(uint32_t c, int k) {
  return static_cast<int>(c << (22 - 10 * k)) >> 22;
}
__device__ __forceinline__ uint32_t pack_cross(int x, int y, int z) {
  const bool sat = x < -511 || x > 511 || y < -511 || y > 511 || z < -511 || z > 511;
  return (static_cast<uint32_t>(x) & 0x3ffu) | ((static_cast<uint32_t>(y) & 0x3ffu) << 10) |
         ((static_cast<uint32_t>(z) & 0x3ffu) << 20) | (sat ? kCrossSaturated : 0u);
}

// Kernels launched as programmatic dependents (launch_dependent) start
// while the previous kernel in the stream drains and wait here, before
// their first read of its results, until it has completed and its writes
// are visible.  Without that launch attribute this returns at once.
__device__ __forceinline__ void wait_prior_grid() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// |d|^2 with the contraction order fixed: fma(dz,dz, fma(dx,dx, dy*dy)), the
// order nvcc gives the reference's dx * dx + dy * dy + dz * dz (its neighbour
// lists include exactly the pairs this form puts at or below the cutoff).
__device__ __forceinline__ float norm2(float dx, float dy, float dz) {
  return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
}

__device__ __forceinline__ uint32_t axis_cell(float x, float lo, float inv,
                                              uint32_t n) {
  const float scaled = __fmul_rn(__fsub_rn(x, lo), inv);
  if (scaled <= 0.0f) return 0u;
  if (scaled >= (float)n) return n - 1u;   // also catches NaN-free overflow
  const uint32_t idx = (uint32_t)scaled;
  return idx >= n ? n - 1u : idx;
}

// Cells visited along one axis around centre c, unique so that one or two
// cells per axis are not visited twice (same set rule as the reference's
// unique_axis_cells, small_dimension_neighbor_builder.cu:56-76): the k-th of
// min(n, 3) cells, computed without an indexed array so the hot loop's state
// stays in registers.
__device__ __forceinline__ uint32_t stencil_cell(uint32_t c, uint32_t n, uint32_t k) {
  if (n < 3u) return k;
  const uint32_t t = c + k + n - 1u;  // c - 1 + k, wrapped
  return t >= n ? (t >= 2u * n ? t - 2u * n : t - n) : t;
}

// Last block of a replica to finish a kernel (threadfence-reduction pattern:
// no waiting, the last arriving block does the per-replica epilogue).
__device__ __forceinline__ bool arrive_last(unsigned int* counter,
                                            unsigned int n_blocks) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned prev = atomicAdd(counter, 1u);
    last = (prev + 1u == n_blocks);
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

}  // namespace bb
