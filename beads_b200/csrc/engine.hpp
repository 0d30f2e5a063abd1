// engine.hpp -- the batched device engine behind the C ABI.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/beads_b200.h"
#include "device.cuh"
#include "kernels.cuh"
#include "setup.hpp"

namespace bb {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct NeighborOverflow : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct NonFinite : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void cuda_check(cudaError_t e, const char* what);

struct ReplicaHost {
  Plan plan;
  uint32_t n_atoms = 0;
  uint32_t atom_begin = 0;
  uint32_t n_pad = 0;
  uint32_t tag_base = 0;
  int units = 0;
  float box_lo[3], box_hi[3];
  uint32_t max_neighbors = 0;
  uint64_t excluded_pairs = 0;
  uint32_t n_bonds = 0, n_angles = 0, n_dihedrals = 0;
  double dt = 0;
  int thermostat = 0;
};

class Engine {
 public:
  Engine(uint32_t n_replicas, const beads_system_desc* systems,
         const beads_forcefield_desc* ffs, const beads_neighbor_desc* nbrs,
         const beads_dynamics_desc* dyns);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  uint32_t n_replicas() const { return static_cast<uint32_t>(rep_.size()); }
  uint64_t n_particles_total() const { return n_tags_; }
  const ReplicaHost& replica(uint32_t r) const { return rep_.at(r); }
  cudaStream_t stream() const { return stream_; }

  // Initial (or explicit) build + force/observable evaluation.
  void eval();
  // Advance `steps`; observables on multiples of obs_every (0 = never).
  // Returns true if the last step was an observable step.
  bool run(uint64_t steps, uint64_t obs_every);
  void minimize(uint32_t iterations, float dmax, float fref);

  void observables(std::vector<beads_observables>& out);
  void state(uint32_t r, float* pos, float* vel, float* force, int32_t* img,
             uint32_t* tag_slot_order = nullptr, int32_t* type_slot = nullptr);
  // Slot-order view of one replica (for trajectory records / snapshots).
  struct SlotView {
    std::vector<float4> pos, vel, force;
    std::vector<int4> img;
    std::vector<uint32_t> tag, mol;
  };
  void slot_view(uint32_t r, SlotView& out);
  void set_state(uint32_t r, const float* pos, const float* vel);
  void upload_all(const float* pos, const float* vel);
  void download_all(float* pos, float* vel);
  void debug_cells(uint32_t r, uint32_t* cell_by_tag);
  void debug_neighbors(uint32_t r, uint32_t cap, uint32_t* counts, uint32_t* partners);
  uint64_t step() const { return step_; }
  bool initialized() const { return initialized_; }
  // Applies a pending Berendsen scale to the velocities (state reads).
  void flush_lambda();
  double profile(int stage, uint32_t reps);
  void list_stats(uint64_t* total, uint32_t* max_count);
  // Completed steps, neighbour builds and dangerous rebuilds of one replica.
  void counters(uint32_t replica, uint64_t out[3]);
  void check_status();

 private:
  template <typename T>
  T* dalloc(size_t count);
  void upload_static(uint32_t n, const beads_system_desc* systems,
                     const beads_forcefield_desc* ffs,
                     const beads_neighbor_desc* nbrs,
                     const beads_dynamics_desc* dyns);
  void record_step(bool observables);
  void record_step_conditional(bool observables);
  cudaGraphExec_t graph_for(uint32_t steps, bool obs_last);
  void launch_chunk(uint32_t steps, bool obs_last);
  void sync();

  std::vector<ReplicaHost> rep_;
  std::vector<void*> allocations_;
  DeviceView v_{};
  StepLaunch launch_{};
  cudaStream_t stream_ = nullptr;
  uint64_t n_tags_ = 0;
  uint64_t step_ = 0;
  bool initialized_ = false;
  bool use_graphs_ = true;
  bool use_conditional_ = true;
  cudaStream_t side_stream_ = nullptr;
  std::map<std::pair<uint32_t, bool>, std::pair<cudaGraph_t, cudaGraphExec_t>> graphs_;
  ReplicaObs* h_obs_ = nullptr;        // pinned
  ReplicaState* h_state_ = nullptr;    // pinned
  float* d_xfer_pos_ = nullptr;        // tag-order staging (lazily allocated)
  float* d_xfer_vel_ = nullptr;
  std::vector<uint32_t> host_row_tag_;  // per replica concatenated (global tag idx)
};

}  // namespace bb
