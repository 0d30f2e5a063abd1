// engine.hpp -- the batched device engine behind the C ABI.
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
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
  int n_types = 0;
  uint32_t lj_offset = 0;        // first entry of the replica's LJ table
  double lj_cutoff = 0;
  int lj_shift = 0;
  uint32_t sort_every = 0;       // reorder cadence in builds (0 = never)
  int n_bond_types = 0, n_angle_types = 0, n_dihedral_types = 0;
  uint32_t bond_type_base = 0, angle_type_base = 0, dihedral_type_base = 0;
};

struct AdjointStore;  // adjoint.cu

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
  //
  // The steps run as captured chunks of at most 16.  After launching chunk
  // k the host reads the status words that chunk k - 1 left (a pinned copy
  // queued behind it, so the device keeps chunk k to work on) and raises the
  // error of a replica whose list overflowed, whose energy left the
  // fixed-point range or whose velocities became non-finite: at most one
  // chunk after the step that failed.  `poll`, when given, is called at the
  // first chunk boundary at or after every `poll_every` steps; a true return
  // stops the run with std::runtime_error("interrupted") once the queued
  // chunks have drained.
  bool run(uint64_t steps, uint64_t obs_every, const std::function<bool()>* poll = nullptr,
           uint64_t poll_every = 1);
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
  // Pair forces from shared-memory cell tiles (list rows by cell order, stage
  // indices as entries) or from global gathers (rows by slot, slot entries).
  // Contexts start staged when some replica qualifies; switching rebuilds the
  // list before the next force evaluation.  Results are the same bits.
  void set_list_staged(bool staged);
  bool list_staged() const { return v_.list_by_q != 0; }
  void debug_neighbors_staged(uint32_t r, uint32_t cap, uint32_t* counts, uint32_t* partners);
  void relayout_list();
  uint64_t step() const { return step_; }
  bool initialized() const { return initialized_; }
  // Applies a pending Berendsen scale to the velocities (state reads).
  void flush_lambda();
  double profile(int stage, uint32_t reps);
  void list_stats(uint64_t* total, uint32_t* max_count);
  // Completed steps, neighbour builds and dangerous rebuilds of one replica,
  // and the launches of the rebuild chain so far (whole batch).
  void counters(uint32_t replica, uint64_t out[4]);
  // Kernels one MD step launches under the current schedule, and the
  // kernels of one rebuild chain when that chain runs only on rebuild steps
  // (0 when every step launches it: no conditional graph node).  Counted
  // as the kernel nodes of one captured step; nothing is executed.
  void launch_counts(uint32_t& per_step, uint32_t& per_chain);
  void check_status();
  // Kernel schedule of the step: threads per particle of the pair-force
  // kernel (1, 2 or 4), its batch depth (4 or 8 list entries in flight per
  // thread), whether its list loads bypass L1, and whether the second
  // half-kick runs inside the last force kernel.  Every choice gives bit-identical results.  tpa = 0 hands
  // the choice back to the autotuner, which times every candidate on this
  // batch at the first run (velocities and step state restored) and keeps
  // the fastest.
  void set_tuning(int tpa, int fuse_post, int unroll, int no_l1);
  void tuning(int* tpa, int* fuse_post, int* unroll, int* no_l1, int* autotuned) const;
  void autotune();

  // ---- adjoint (reverse-mode gradients of a trajectory; adjoint.cu) ----
  // Replaces the LJ eps/sigma tables of one replica (full n_types^2 tables).
  void set_lj(uint32_t replica, const double* eps, const double* sigma);
  // Replaces one replica's harmonic bonded parameters (NULL: unchanged);
  // angle theta0 in degrees as in beads_forcefield_desc.
  void set_bonded(uint32_t replica, const double* bond_k, const double* bond_r0,
                  const double* angle_k, const double* angle_theta0_deg,
                  const double* dihedral_k);
  // Runs `steps` velocity-Verlet steps from the current state (forces and
  // the list are rebuilt first, as a fresh run), keeping a checkpoint every
  // `checkpoint_every` steps (0: keep every step, no replay later).  obs receives [step - record_from][replica]
  // {pair+bonded PE, virial, thermo KE} for steps record_from..steps.
  void adjoint_forward(uint64_t steps, uint64_t record_from, uint32_t checkpoint_every,
                       double* obs);
  // Given dL/d(obs) in the same layout, returns dL/d(eps), dL/d(sigma)
  // ([replica][n_types^2] each, per ordered type pair of the table), dL/dx0
  // and dL/dv0 (tag order, [n_particles_total][3]).  The particle state is
  // the end-of-forward state again afterwards.
  void adjoint_backward(const double* obs_grad, double* grad_eps, double* grad_sigma,
                        float* grad_pos, float* grad_vel);
  // Bonded parameter gradients of the last adjoint_backward, by global type
  // (replicas' types in batch order): bonds [k, r0], angles [k, theta0 per
  // degree], dihedrals [k].
  void adjoint_bonded_grads(double* grad_bond, double* grad_angle, double* grad_dihedral);
  uint32_t n_bond_types_total() const { return total_bond_types_; }
  uint32_t n_angle_types_total() const { return total_angle_types_; }
  uint32_t n_dihedral_types_total() const { return total_dihedral_types_; }

 private:
  // Switches the periodic slot reorder off (false) or back to each replica's
  // own cadence (true); adjoint runs need fixed slots.
  void set_sort_enabled(bool on);
  void adjoint_restore(uint32_t segment);
  void adjoint_record(uint32_t k);
  void adjoint_snapshot(uint32_t k, bool all);
  void adjoint_segment_storage(uint32_t K);
  void adjoint_select_list(uint32_t a, uint32_t m, std::vector<int>& current,
                           const std::vector<uint32_t>& flags);
  std::unique_ptr<AdjointStore> adj_;
  void clear_graphs();
  template <typename T>
  T* dalloc(size_t count);
  void upload_static(uint32_t n, const beads_system_desc* systems,
                     const beads_forcefield_desc* ffs,
                     const beads_neighbor_desc* nbrs,
                     const beads_dynamics_desc* dyns);
  void record_step(bool observables);
  void record_step_conditional(bool observables);
  cudaGraphExec_t graph_for(uint32_t steps, bool obs_last);
  // Adjoint: one captured graph per segment length replays the segment's
  // steps with their recording (adjoint.cu).
  cudaGraphExec_t replay_graph_for(uint32_t steps);
  void clear_replay_graphs();
  void launch_chunk(uint32_t steps, bool obs_last);
  void sync();
  // Host<->device copies ordered on stream_ and complete on return.  The
  // engine stream is non-blocking, so a plain cudaMemcpy (legacy stream) is
  // not ordered against its kernels or its zero fills.
  void h2d(void* dst, const void* src, size_t bytes, const char* what);
  void d2h(void* dst, const void* src, size_t bytes, const char* what);

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
  cudaGraph_t last_chain_body_ = nullptr;  // body of the last recorded conditional node
  uint32_t total_bond_types_ = 0, total_angle_types_ = 0, total_dihedral_types_ = 0;
  bool staged_ = false;                // some replica stages its pair forces
  uint32_t stage_cap_ = 0;             // stage entries per group (k_lj_staged)
  bool tuning_fixed_ = false;          // set_tuning() with an explicit choice
  bool layout_fixed_ = false;          // set_list_staged() called: the autotuner keeps the layout
  bool any_sparse_ = false, any_dense_ = false;  // list build forms in use (k_build_sparse / k_build)
  float4* relayout_pos_ = nullptr;     // relayout_list save buffers (allocated at first use)
  int4* relayout_img_ = nullptr;
  uint32_t* relayout_cross_ = nullptr;
  bool tuned_ = false;                 // autotune() has run
  cudaStream_t side_stream_ = nullptr;
  std::map<std::pair<uint32_t, bool>, std::pair<cudaGraph_t, cudaGraphExec_t>> graphs_;
  std::map<uint32_t, std::pair<cudaGraph_t, cudaGraphExec_t>> replay_graphs_;
  ReplicaObs* h_obs_ = nullptr;        // pinned
  ReplicaState* h_state_ = nullptr;    // pinned
  // Status words of the last kStatusRing chunks (pinned, [kStatusRing][n_replicas]).
  // The run loop checks a chunk's words once the two chunks after it are
  // queued, so the GPU keeps two chunks of work while the host waits.
  static constexpr uint32_t kStatusRing = 3;
  unsigned* h_chunk_status_ = nullptr;
  cudaEvent_t chunk_event_[kStatusRing] = {};
  float* d_xfer_pos_ = nullptr;        // tag-order staging (lazily allocated)
  float* d_xfer_vel_ = nullptr;
  std::vector<uint32_t> host_row_tag_;  // per replica concatenated (global tag idx)
};

}  // namespace bb
