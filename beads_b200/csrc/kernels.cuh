// kernels.cuh -- launch interface of the per-step kernels.
#pragma once

#include "device.cuh"

namespace bb {

// One MD step is: pre (Berendsen lambda of the previous step, half-kick,
// drift, wrap, displacement check, rebuild decision) -> rebuild chain (each
// kernel returns at once for replicas that do not rebuild) -> pair forces ->
// bonded forces -> post (half-kick, kinetic energy, observables, next lambda).
enum PreMode : int { kPreVerlet = 0, kPreDescent = 1 };

struct StepLaunch {
  DeviceView v;
  cudaStream_t stream;
  uint32_t max_cells_per_replica;
  uint32_t max_atoms_per_replica;
  int excl_cap;           // 0, 4, 8, 16, 32 or 64
  int lj_tpa;             // threads per particle of the pair-force kernel: 1, 2, 4
  int lj_unroll;          // list entries in flight per thread and batch: 4 or 8
  int lj_no_l1;           // list entries loaded without allocating L1 lines
  int lj_types;           // largest LJ table side over the batch (1, 2: specialised)
  int fuse_post;          // second half-kick inside the last force kernel
  int need_kinetic;       // a thermostat is active in some replica
  int any_dense;          // some replica builds its lists a warp per cell (k_build)
  int any_sparse;         // some replica builds them a thread per particle
  uint32_t chain_grid;    // blocks of the chain's per-slot kernels with the block list
  float sd_dmax;          // descent: displacement cap
  float sd_fref;          // descent: force floor
};

// use_cond: the launch is captured in front of a conditional graph node whose
// handle is `cond`; the kernel switches that node on when a replica rebuilds.
void launch_pre(const StepLaunch& l, int mode, cudaGraphConditionalHandle cond = 0,
                bool use_cond = false);
// force_all: every replica rebuilds now; count_build = false rebuilds without
// counting a build or reordering (a list-layout change of the same list).
void launch_rebuild(const StepLaunch& l, bool force_all, bool count_build = true);
// post: finish the step with the second half-kick, the kinetic-energy total
// and the per-replica step epilogue -- inside the last force kernel when
// fuse_post is set, else as a separate k_post launch.
// parts: which force kernels run (kForcePair | kForceBonded; the profiler
// times them one at a time).
constexpr int kForcePair = 1, kForceBonded = 2;
void launch_forces(const StepLaunch& l, bool observables, bool clamp, bool post = false,
                   int parts = kForcePair | kForceBonded);
void launch_post(const StepLaunch& l, bool kick, bool observables);
// Staged contexts (list rows by cell order): raise the dynamic shared-memory
// limit of the staged pair-force kernels, and decode the list into slot rows
// of neighbour slots (debug views).
void prepare_staged_kernels(size_t smem);
void launch_list_to_slots(const StepLaunch& l, uint32_t cap, uint32_t* out_count, uint32_t* out);
void launch_project_exclusions(const StepLaunch& l, bool force_all);
void launch_apply_lambda(const StepLaunch& l);
// Scatter a tag-ordered host copy (already on the device) into slots.
void launch_scatter_state(const StepLaunch& l, const float* pos_tag,
                          const float* vel_tag, uint32_t n_tags_total);
void launch_gather_state(const StepLaunch& l, float* pos_tag, float* vel_tag,
                         uint32_t n_tags_total);

}  // namespace bb
