// adjoint.hpp -- device storage of the reverse-mode (adjoint) pass.
//
// The forward pass keeps checkpoints of the full step state every K steps
// (and one of the final state); the backward pass replays one segment at a
// time from its checkpoint, recording positions, velocities, Berendsen scales
// and kinetic energies of every step of the segment, then walks the segment
// backwards.  Memory: (segments + 1) checkpoints of 80 bytes per slot plus
// K + 1 recorded steps of 32 bytes per slot; when the device has room, K + 1
// list snapshots of 4 (max_neighbors + 1) bytes per slot, so the reverse
// sweep reads each step's list instead of rebuilding it.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "device.cuh"

namespace bb {

struct AdjointStore {
  uint64_t steps = 0;         // T
  uint64_t record_from = 0;   // first step whose observables enter the loss
  uint32_t every = 0;         // K
  uint32_t segments = 0;      // ceil(T / K)
  uint32_t slots = 0;         // S
  uint32_t replicas = 0;      // R
  int max_types = 0;          // LJ table side of the largest replica table
  bool forward_done = false;
  bool store_all = false;     // every step kept by the forward pass (no replay)
  cudaStream_t stream = nullptr;  // the engine stream: zero fills are ordered on it

  // checkpoints: segment starts 0..segments-1, then the final state
  float4* ck_pos = nullptr;
  float4* ck_vel = nullptr;
  int4* ck_img = nullptr;
  float4* ck_ref_pos = nullptr;
  int4* ck_ref_img = nullptr;
  std::vector<ReplicaState> ck_state;
  uint64_t ck_capacity = 0;   // checkpoints allocated

  // one replayed segment: steps a..a+K
  float4* seg_pos = nullptr;
  float4* seg_vel = nullptr;
  double* seg_lam = nullptr;     // [k * R + r] Berendsen scale after step a+k
  double* seg_kin = nullptr;     // [k * R + r] kinetic energy after step a+k
  uint32_t* seg_flags = nullptr; // [k * R + r] replica rebuilt its list at step a+k
  int* seg_src = nullptr;        // [k * R + r] step whose positions built step a+k's list
  uint32_t* seg_changed = nullptr;  // [k * R + r] that list differs from step a+k+1's
  uint32_t seg_capacity = 0;     // K + 1 allocated

  // list snapshots of one replayed segment: snapshot 0 holds every replica's
  // list at the segment start, snapshot k the rows of the replicas that
  // rebuilt at step a+k (the other rows of snapshot k are not used)
  uint32_t* snap_nbr = nullptr;  // [k][slots * stride], the list layout of DeviceView::nbr
  uint32_t* snap_cnt = nullptr;  // [k][slots]
  uint32_t snap_capacity = 0;    // snapshots allocated (0: lists are rebuilt)
  bool snap_on = false;          // the current backward pass uses the snapshots

  // adjoint vectors (per slot) and reductions
  float4* xbar = nullptr;
  float4* vbar = nullptr;
  float4* fbar = nullptr;
  float4* ubar = nullptr;
  double* obs_grad = nullptr;    // [(T + 1) * R * 3]
  uint64_t obs_capacity = 0;
  long long* theta = nullptr;    // [R][types^2][eps, sigma][whole, frac]
  float* tag_xfer = nullptr;     // [3 * particles] tag-order staging
  int* shift_on = nullptr;       // [R] LJ energy shift active
  long long* dot = nullptr;          // [2][R][2] sum u_bar . v (fixed point)
  long long* theta_bond = nullptr;   // [bond types][k, r0][2]
  long long* theta_angle = nullptr;  // [angle types][k, theta0][2]
  long long* theta_dihedral = nullptr;  // [dihedral types][2]

  std::vector<void*> allocations;
  ~AdjointStore();
  template <typename T>
  T* alloc(size_t count);
};

}  // namespace bb
