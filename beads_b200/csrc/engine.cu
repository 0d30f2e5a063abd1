// engine.cu -- host side of the batched device engine: memory layout, static
// tables, the captured step loop and host transfers.
#include "engine.hpp"
#include "adjoint.hpp"
#include "trace.hpp"

#include <cstdio>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <sstream>

namespace bb {

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    throw CudaError(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
  }
}

namespace {

constexpr uint32_t kChunkMax = 16;     // steps per captured graph
constexpr double kKbNmKjMol = 0.00831446261815324;
constexpr double kPressNmKjMol = 16.60539067;

uint32_t round_up(uint32_t x, uint32_t m) { return (x + m - 1) / m * m; }

int exclusion_capacity(uint32_t degree) {
  if (degree == 0) return 0;
  for (int cap : {4, 8, 16, 32, 64}) {
    if (degree <= static_cast<uint32_t>(cap)) return cap;
  }
  throw InvalidArgument(
      "bonded exclusions with more than 64 partners per particle are not supported.");
}

}  // namespace

template <typename T>
T* Engine::dalloc(size_t count) {
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cuda_check(cudaMalloc(&p, bytes), "cudaMalloc");
  allocations_.push_back(p);
  cuda_check(cudaMemsetAsync(p, 0, bytes, stream_), "cudaMemset");
  return static_cast<T*>(p);
}

Engine::Engine(uint32_t n, const beads_system_desc* systems,
               const beads_forcefield_desc* ffs, const beads_neighbor_desc* nbrs,
               const beads_dynamics_desc* dyns) {
  if (n == 0) throw InvalidArgument("a batch needs at least one replica.");
  // BEADS_GRAPHS=0 launches every kernel directly (same kernels, no graph):
  // profilers that cannot see kernels inside conditional graphs need it.
  if (const char* g = std::getenv("BEADS_GRAPHS")) use_graphs_ = std::string(g) != "0";
  for (uint32_t r = 0; r < n; ++r) validate_replica(systems[r], ffs[r], nbrs[r], dyns[r]);
  cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream create");
  try {
    upload_static(n, systems, ffs, nbrs, dyns);
  } catch (...) {
    for (void* p : allocations_) cudaFree(p);
    allocations_.clear();
    if (h_obs_) cudaFreeHost(h_obs_);
    if (h_state_) cudaFreeHost(h_state_);
    cudaStreamDestroy(stream_);
    throw;
  }
  // BEADS_SCHEDULE="tpa,fuse_post,depth,list_bypass_l1" fixes the kernel
  // schedule for every context of the process (reproducible profiling, no
  // autotuning); results do not depend on it.
  if (const char* e = std::getenv("BEADS_SCHEDULE")) {
    int t = 0, f = 0, u = 0, b = 0;
    if (std::sscanf(e, "%d,%d,%d,%d", &t, &f, &u, &b) == 4 && t != 0) set_tuning(t, f, u, b);
  }
}

void Engine::set_sort_enabled(bool on) {
  sync();
  for (uint32_t r = 0; r < rep_.size(); ++r) {
    const uint32_t value = on ? rep_[r].sort_every : 0u;
    ReplicaParams* dst = const_cast<ReplicaParams*>(v_.rp) + r;
    h2d(&dst->sort_every, &value, sizeof(value), "sort cadence");
  }
}

void Engine::clear_graphs() {
  if (stream_) cudaStreamSynchronize(stream_);
  for (auto& kv : graphs_) {
    cudaGraphExecDestroy(kv.second.second);
    cudaGraphDestroy(kv.second.first);
  }
  graphs_.clear();
  clear_replay_graphs();
}

void Engine::clear_replay_graphs() {
  if (stream_) cudaStreamSynchronize(stream_);
  for (auto& kv : replay_graphs_) {
    cudaGraphExecDestroy(kv.second.second);
    cudaGraphDestroy(kv.second.first);
  }
  replay_graphs_.clear();
}

void Engine::set_tuning(int tpa, int fuse_post, int unroll, int no_l1) {
  if (tpa == 0) {
    tuning_fixed_ = false;
    tuned_ = false;
    return;
  }
  if (tpa != 1 && tpa != 2 && tpa != 4) throw InvalidArgument("threads per particle must be 1, 2 or 4.");
  if (unroll != 4 && unroll != 8) throw InvalidArgument("batch depth must be 4 or 8.");
  clear_graphs();
  launch_.lj_tpa = tpa;
  launch_.lj_unroll = unroll;
  launch_.lj_no_l1 = no_l1 ? 1 : 0;
  launch_.fuse_post = fuse_post ? 1 : 0;
  tuning_fixed_ = true;
}

void Engine::tuning(int* tpa, int* fuse_post, int* unroll, int* no_l1, int* autotuned) const {
  *tpa = launch_.lj_tpa;
  *fuse_post = launch_.fuse_post;
  *unroll = launch_.lj_unroll;
  *no_l1 = launch_.lj_no_l1;
  *autotuned = (tuned_ && !tuning_fixed_) ? 1 : 0;
}

// Times the force stage of a step (pair forces, bonded terms, second
// half-kick and kinetic total) under every schedule on the current list and
// keeps the fastest.  The kicks of the trial launches are undone.  With
// BEADS_TUNE_LOG=1 the timings go to stderr.
void Engine::autotune() {
  TraceRange trace("beads.autotune");
  if (!initialized_) eval();
  constexpr int kWarm = 1, kReps = 4;
  const bool log = [] {
    const char* e = std::getenv("BEADS_TUNE_LOG");
    return e && std::string(e) == "1";
  }();
  std::vector<ReplicaState> saved(rep_.size());
  sync();
  d2h(saved.data(), v_.rs, saved.size() * sizeof(ReplicaState), "state save");
  cuda_check(cudaMemcpyAsync(v_.vel2, v_.vel, v_.n_slots * sizeof(float4),
                             cudaMemcpyDeviceToDevice, stream_), "velocity save");
  cudaEvent_t a = nullptr, b = nullptr;
  cuda_check(cudaEventCreate(&a), "event create");
  cuda_check(cudaEventCreate(&b), "event create");
  float best = 0.f;
  StepLaunch chosen = launch_;
  auto trial = [&](const StepLaunch& l) {
    for (int k = 0; k < kWarm; ++k) launch_forces(l, false, false, true);
    cuda_check(cudaEventRecord(a, stream_), "event record");
    for (int k = 0; k < kReps; ++k) launch_forces(l, false, false, true);
    cuda_check(cudaEventRecord(b, stream_), "event record");
    cuda_check(cudaEventSynchronize(b), "event sync");
    float ms = 0.f;
    cuda_check(cudaEventElapsedTime(&ms, a, b), "event elapsed");
    if (log) {
      std::fprintf(stderr, "beads autotune: tpa %d depth %d no_l1 %d fuse_post %d: %.4f ms\n",
                   l.lj_tpa, l.lj_unroll, l.lj_no_l1, l.fuse_post, ms / kReps);
    }
    if (best == 0.f || ms < best) {
      best = ms;
      chosen = l;
    }
  };
  // One coordinate at a time, each from the best so far: threads per
  // particle {1, 2, 4} at batch depth 4 with list loads bypassing L1, then
  // depth 8, then list loads through L1 (the staged kernel reads its
  // neighbour positions from shared memory and has no L1 choice), then the
  // second half-kick fused into the force kernel: six trials per layout
  // instead of the full grid of thirteen, which a short run pays for.
  auto tune_layout = [&]() {
    best = 0.f;
    const bool staged_now = v_.list_by_q != 0;
    for (int tpa : {1, 2, 4}) {
      StepLaunch l = launch_;
      l.lj_tpa = tpa;
      l.lj_unroll = 4;
      l.lj_no_l1 = 1;
      l.fuse_post = 0;
      trial(l);
    }
    StepLaunch deeper = chosen;
    deeper.lj_unroll = 8;
    trial(deeper);
    if (!staged_now) {
      StepLaunch l1 = chosen;
      l1.lj_no_l1 = 0;
      trial(l1);
    }
    StepLaunch fused = chosen;
    fused.fuse_post = 1;
    trial(fused);
  };
  try {
    tune_layout();
    // Both list layouts when the context can stage: the other layout is
    // built from the same positions (relayout_list) and tuned the same way.
    if (stage_cap_ > 0 && !layout_fixed_) {
      const float best_first = best;
      const StepLaunch chosen_first = chosen;
      const bool first_staged = v_.list_by_q != 0;
      v_.list_by_q = first_staged ? 0 : 1;
      launch_.v = v_;
      relayout_list();
      tune_layout();
      if (log) {
        std::fprintf(stderr, "beads autotune: staged layout %.4f ms, slot layout %.4f ms\n",
                     (first_staged ? best_first : best) / kReps,
                     (first_staged ? best : best_first) / kReps);
      }
      if (best_first <= best) {
        best = best_first;
        chosen = chosen_first;
        v_.list_by_q = first_staged ? 1 : 0;
        launch_.v = v_;
        relayout_list();
      }
    }
  } catch (...) {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    throw;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cuda_check(cudaMemcpyAsync(v_.vel, v_.vel2, v_.n_slots * sizeof(float4),
                             cudaMemcpyDeviceToDevice, stream_), "velocity restore");
  cuda_check(cudaMemcpyAsync(v_.rs, saved.data(), saved.size() * sizeof(ReplicaState),
                             cudaMemcpyHostToDevice, stream_), "state restore");
  sync();
  // Captured graphs hold the kernels of one schedule and one layout.
  clear_graphs();
  launch_.lj_tpa = chosen.lj_tpa;
  launch_.lj_unroll = chosen.lj_unroll;
  launch_.lj_no_l1 = chosen.lj_no_l1;
  launch_.fuse_post = chosen.fuse_post;
  tuned_ = true;
}

Engine::~Engine() {
  if (stream_) cudaStreamSynchronize(stream_);
  for (auto& kv : graphs_) {
    cudaGraphExecDestroy(kv.second.second);
    cudaGraphDestroy(kv.second.first);
  }
  for (auto& kv : replay_graphs_) {
    cudaGraphExecDestroy(kv.second.second);
    cudaGraphDestroy(kv.second.first);
  }
  for (void* p : allocations_) cudaFree(p);
  if (h_obs_) cudaFreeHost(h_obs_);
  if (h_state_) cudaFreeHost(h_state_);
  if (h_chunk_status_) cudaFreeHost(h_chunk_status_);
  for (cudaEvent_t e : chunk_event_) {
    if (e) cudaEventDestroy(e);
  }
  if (side_stream_) cudaStreamDestroy(side_stream_);
  if (stream_) cudaStreamDestroy(stream_);
}

void Engine::upload_static(uint32_t n, const beads_system_desc* systems,
                           const beads_forcefield_desc* ffs,
                           const beads_neighbor_desc* nbrs,
                           const beads_dynamics_desc* dyns) {
  rep_.resize(n);
  uint64_t slots = 0, tags = 0, cells = 0, lj_entries = 0;
  uint64_t bonds = 0, angles = 0, dihedrals = 0;
  uint32_t bond_types = 0, angle_types = 0, dihedral_types = 0;
  uint32_t stride = 0, max_cells = 0, max_atoms = 0, max_degree = 0;
  bool any_bonded = false, any_thermostat = false;

  // Exclusion partner lists per replica (global tag indices).
  std::vector<std::vector<uint32_t>> excl_partners;  // by global tag
  std::vector<ReplicaParams> rp(n);
  for (uint32_t r = 0; r < n; ++r) {
    const beads_system_desc& s = systems[r];
    const beads_forcefield_desc& f = ffs[r];
    ReplicaHost& h = rep_[r];
    h.plan = make_plan(s.box_lo, s.box_hi, f.lj_cutoff, nbrs[r].cutoff_buffer);
    h.n_atoms = s.n_particles;
    h.atom_begin = static_cast<uint32_t>(slots);
    h.n_pad = round_up(s.n_particles, kBlock);
    h.tag_base = static_cast<uint32_t>(tags);
    h.units = s.units;
    std::memcpy(h.box_lo, s.box_lo, sizeof(h.box_lo));
    std::memcpy(h.box_hi, s.box_hi, sizeof(h.box_hi));
    h.max_neighbors = nbrs[r].max_neighbors;
    h.n_bonds = s.n_bonds;
    h.n_angles = s.n_angles;
    h.n_dihedrals = s.n_dihedrals;
    h.dt = dyns[r].dt;
    h.thermostat = dyns[r].thermostat;
    h.n_types = f.n_types;
    h.lj_cutoff = f.lj_cutoff;
    h.lj_shift = f.lj_shift;
    slots += h.n_pad;
    tags += s.n_particles;
    if (slots > 0xF0000000ull) throw OverflowError("total particle slots exceed index range.");
    stride = std::max(stride, h.max_neighbors);
    max_cells = std::max(max_cells, h.plan.n_cells);
    max_atoms = std::max(max_atoms, h.n_atoms);
    any_bonded |= (s.n_bonds + s.n_angles + s.n_dihedrals) > 0;
    any_thermostat |= dyns[r].thermostat == 1;

    ReplicaParams& p = rp[r];
    std::memset(&p, 0, sizeof(p));
    for (int a = 0; a < 3; ++a) {
      p.lo[a] = s.box_lo[a];
      p.len[a] = s.box_hi[a] - s.box_lo[a];
      p.half[a] = 0.5f * p.len[a];
      p.inv_len[a] = 1.0f / p.len[a];
      p.nc[a] = h.plan.nc[a];
      p.inv_cell[a] = h.plan.inv_cell[a];
    }
    p.atom_begin = h.atom_begin;
    p.n_atoms = h.n_atoms;
    p.n_pad = h.n_pad;
    p.block_begin = h.atom_begin / kBlock;
    p.tag_base = h.tag_base;
    p.cell_begin = static_cast<uint32_t>(cells);
    p.start_base = static_cast<uint32_t>(cells + r);
    p.n_cells = h.plan.n_cells;
    cells += h.plan.n_cells;
    p.search_cut_sq = h.plan.search_cutoff_sq;
    p.force_cut_sq = h.plan.force_cutoff_sq;
    const float half_skin = 0.5f * h.plan.cutoff_buffer;
    p.disp_thr_sq = half_skin * half_skin;
    p.skin = h.plan.cutoff_buffer;
    p.max_neighbors = h.max_neighbors;
    p.check_every = static_cast<uint32_t>(std::min<uint64_t>(nbrs[r].rebuild_check_every, 0xFFFFFFFFull));
    // The reference's direct path never reorders particles (neighbor_system.cpp:113-119).
    p.sort_every = h.plan.path == kPathDirect
                       ? 0u
                       : static_cast<uint32_t>(std::min<uint64_t>(nbrs[r].sort_every_rebuild, 0xFFFFFFFFull));
    h.sort_every = p.sort_every;
    p.dt = static_cast<float>(dyns[r].dt);
    p.thermostat = dyns[r].thermostat;
    p.kb = s.units == BEADS_UNITS_NM_KJMOL ? kKbNmKjMol : 1.0;
    p.press_scale = s.units == BEADS_UNITS_NM_KJMOL ? kPressNmKjMol : 1.0;
    p.kt_target = p.kb * static_cast<double>(static_cast<float>(dyns[r].temperature));
    p.tau = static_cast<double>(static_cast<float>(dyns[r].tau));
    const double dof = 3.0 * static_cast<double>(s.n_particles) - 3.0;
    p.dof = dof > 0.0 ? dof : 0.0;
    p.volume = static_cast<double>(p.len[0]) * p.len[1] * p.len[2];
    p.lj_offset = static_cast<uint32_t>(lj_entries);
    rep_[r].lj_offset = p.lj_offset;
    p.n_types = f.n_types;
    lj_entries += static_cast<uint64_t>(f.n_types) * f.n_types;
    p.bond_type_base = bond_types;
    p.angle_type_base = angle_types;
    p.dihedral_type_base = dihedral_types;
    rep_[r].bond_type_base = bond_types;
    rep_[r].angle_type_base = angle_types;
    rep_[r].dihedral_type_base = dihedral_types;
    rep_[r].n_bond_types = f.n_bond_types;
    rep_[r].n_angle_types = f.n_angle_types;
    rep_[r].n_dihedral_types = f.n_dihedral_types;
    bond_types += f.n_bond_types;
    angle_types += f.n_angle_types;
    dihedral_types += f.n_dihedral_types;
    bonds += s.n_bonds;
    angles += s.n_angles;
    dihedrals += s.n_dihedrals;
  }
  // Cell-tile staging of the pair forces (kernels.cu, stage_layout): a
  // replica with >= 4 cells on every axis stages its groups of 128 particles.
  // A group's stage is 9 stencil rows of the home cells plus one cell on each
  // side per home row: about 9 (128 + 5 m) entries for m particles per cell
  // when the group spans two rows; the capacity adds a quarter for density
  // fluctuations (a group beyond it keeps slot entries).  Replicas that would
  // need more than kStageMaxEntries (crowded cells) are not staged.
  // BEADS_STAGED=0 turns staging off for every context of the process.
  {
    constexpr uint32_t kStageMaxEntries = 8192;  // 128 KiB of shared memory
    bool enabled = true;
    if (const char* e = std::getenv("BEADS_STAGED")) enabled = std::string(e) != "0";
    uint32_t cap = 0;
    for (uint32_t r = 0; r < n; ++r) {
      const ReplicaHost& h = rep_[r];
      const bool regular = h.plan.nc[0] >= 4 && h.plan.nc[1] >= 4 && h.plan.nc[2] >= 4;
      const double occ = static_cast<double>(h.n_atoms) / std::max<uint32_t>(1, h.plan.n_cells);
      const double need = 1.25 * 9.0 * (static_cast<double>(kBlock) + 5.0 * occ);
      const uint32_t want = static_cast<uint32_t>((std::ceil(need) + 255.0) / 256.0) * 256u;
      rp[r].staged = (enabled && regular && want <= kStageMaxEntries) ? 1u : 0u;
      if (rp[r].staged) cap = std::max(cap, want);
    }
    stage_cap_ = cap;
    staged_ = cap > 0;
  }
  // List build form per replica: a thread per particle (k_build_sparse) when
  // its cells hold fewer than kSparseOccupancy particles on average, else a
  // warp per cell (k_build); both write the same lists.  BEADS_BUILD=dense or
  // =sparse forces one form for every replica of the process.
  {
    constexpr double kSparseOccupancy = 8.0;
    std::string force;
    if (const char* e = std::getenv("BEADS_BUILD")) force = e;
    any_sparse_ = any_dense_ = false;
    for (uint32_t r = 0; r < n; ++r) {
      const ReplicaHost& h = rep_[r];
      const double occ = static_cast<double>(h.n_atoms) / std::max<uint32_t>(1, h.plan.n_cells);
      bool sparse = occ < kSparseOccupancy;
      if (force == "dense") sparse = false;
      if (force == "sparse") sparse = true;
      rp[r].sparse = sparse ? 1u : 0u;
      any_sparse_ |= sparse;
      any_dense_ |= !sparse;
    }
  }
  n_tags_ = tags;
  total_bond_types_ = static_cast<uint32_t>(bond_types);
  total_angle_types_ = static_cast<uint32_t>(angle_types);
  total_dihedral_types_ = static_cast<uint32_t>(dihedral_types);
  const uint32_t S = static_cast<uint32_t>(slots);
  const uint32_t T = static_cast<uint32_t>(tags);
  const uint32_t C = static_cast<uint32_t>(cells);
  const uint64_t list_entries = static_cast<uint64_t>(S) * stride;
  if (list_entries > (1ull << 36)) throw OverflowError("NeighborList slot count overflows.");

  // ---- exclusions (tag space) ----
  std::vector<uint32_t> excl_off(T + 1, 0);
  std::vector<uint32_t> excl_tag;
  {
    std::vector<std::vector<uint32_t>> partners(T);
    for (uint32_t r = 0; r < n; ++r) {
      const beads_system_desc& s = systems[r];
      const int d = ffs[r].exclusion_distance;
      if (d <= 0 || s.n_bonds == 0) continue;
      const auto pairs = bond_graph_exclusions(s.n_particles, s.bonds, s.n_bonds, d);
      rep_[r].excluded_pairs = pairs.size();
      const uint32_t base = rep_[r].tag_base;
      for (const auto& pr : pairs) {
        partners[base + pr.first - 1].push_back(base + pr.second - 1);
        partners[base + pr.second - 1].push_back(base + pr.first - 1);
      }
    }
    for (uint32_t t = 0; t < T; ++t) {
      std::sort(partners[t].begin(), partners[t].end());
      max_degree = std::max<uint32_t>(max_degree, static_cast<uint32_t>(partners[t].size()));
      excl_off[t + 1] = excl_off[t] + static_cast<uint32_t>(partners[t].size());
    }
    excl_tag.reserve(excl_off[T]);
    for (uint32_t t = 0; t < T; ++t) {
      excl_tag.insert(excl_tag.end(), partners[t].begin(), partners[t].end());
    }
  }
  const int excl_cap = exclusion_capacity(max_degree);
  for (uint32_t r = 0; r < n; ++r) rp[r].excl_degree = max_degree;

  // ---- particles in input order ----
  // One slot past the last holds the far particle that pads neighbour
  // batches in the pair-force kernel (its distance to every particle is
  // beyond any cutoff).
  std::vector<float4> h_pos(S + 1), h_vel(S);
  h_pos[S] = make_float4(kFarCoord, kFarCoord, kFarCoord, 0.f);
  std::vector<int4> h_img(S);
  std::vector<uint32_t> h_tag(S, 0xffffffffu), h_mol(S, 0), slot_of_tag(T, 0);
  std::vector<uint32_t> block_replica(S / kBlock);
  for (uint32_t r = 0; r < n; ++r) {
    const beads_system_desc& s = systems[r];
    const ReplicaHost& h = rep_[r];
    const std::vector<uint32_t> rt = row_tags(s);
    for (uint32_t k = 0; k < h.n_pad; ++k) {
      const uint32_t slot = h.atom_begin + k;
      if (k < h.n_atoms) {
        int ty = s.types[k] - 1;
        float w;
        std::memcpy(&w, &ty, sizeof(w));
        h_pos[slot] = make_float4(s.positions[3 * k], s.positions[3 * k + 1],
                                  s.positions[3 * k + 2], w);
        const float m = s.masses ? s.masses[k] : 1.0f;
        if (s.velocities) {
          h_vel[slot] = make_float4(s.velocities[3 * k], s.velocities[3 * k + 1],
                                    s.velocities[3 * k + 2], m);
        } else {
          h_vel[slot] = make_float4(0.f, 0.f, 0.f, m);
        }
        h_img[slot] = s.images ? make_int4(s.images[3 * k], s.images[3 * k + 1],
                                           s.images[3 * k + 2], 0)
                               : make_int4(0, 0, 0, 0);
        const uint32_t gt = h.tag_base + rt[k] - 1;
        h_tag[slot] = gt;
        h_mol[slot] = s.molecule_ids ? s.molecule_ids[k] : 1u;
        slot_of_tag[gt] = slot;
      } else {
        h_pos[slot] = make_float4(s.box_lo[0], s.box_lo[1], s.box_lo[2], 0.f);
        h_vel[slot] = make_float4(0.f, 0.f, 0.f, 1.f);
        h_img[slot] = make_int4(0, 0, 0, 0);
      }
    }
    for (uint32_t b = 0; b < h.n_pad / kBlock; ++b) block_replica[h.atom_begin / kBlock + b] = r;
  }

  // ---- bonded tables (global tag indices, global type indices) ----
  std::vector<uint4> h_bonds, h_angles, h_dihedrals;
  std::vector<uint32_t> h_dih_type;
  std::vector<BondCoeff> h_bc;
  std::vector<AngleCoeff> h_ac;
  std::vector<DihedralCoeff> h_dc;
  std::vector<std::vector<uint32_t>> member(T);
  for (uint32_t r = 0; r < n; ++r) {
    const beads_system_desc& s = systems[r];
    const beads_forcefield_desc& f = ffs[r];
    const uint32_t base = rep_[r].tag_base;
    for (int t = 0; t < f.n_bond_types; ++t) {
      h_bc.push_back(BondCoeff{static_cast<float>(f.bond_k[t]), static_cast<float>(f.bond_r0[t])});
    }
    for (int t = 0; t < f.n_angle_types; ++t) {
      const float theta0 = static_cast<float>(f.angle_theta0_deg[t]);
      h_ac.push_back(AngleCoeff{static_cast<float>(f.angle_k[t]),
                                theta0 * 3.14159265358979323846f / 180.0f});
    }
    for (int t = 0; t < f.n_dihedral_types; ++t) {
      h_dc.push_back(DihedralCoeff{static_cast<float>(f.dihedral_k[t]), f.dihedral_d[t],
                                   f.dihedral_n[t], 0});
    }
    for (uint32_t k = 0; k < s.n_bonds; ++k) {
      const uint32_t* b = s.bonds + 3 * (size_t)k;
      const uint32_t idx = static_cast<uint32_t>(h_bonds.size());
      h_bonds.push_back(make_uint4(base + b[0] - 1, base + b[1] - 1,
                                   rp[r].bond_type_base + b[2] - 1, 0));
      member[base + b[0] - 1].push_back(term_pack(kTermBond, 0, idx));
      member[base + b[1] - 1].push_back(term_pack(kTermBond, 1, idx));
    }
    for (uint32_t k = 0; k < s.n_angles; ++k) {
      const uint32_t* a = s.angles + 4 * (size_t)k;
      const uint32_t idx = static_cast<uint32_t>(h_angles.size());
      h_angles.push_back(make_uint4(base + a[0] - 1, base + a[1] - 1, base + a[2] - 1,
                                    rp[r].angle_type_base + a[3] - 1));
      for (uint32_t m = 0; m < 3; ++m) member[base + a[m] - 1].push_back(term_pack(kTermAngle, m, idx));
    }
    for (uint32_t k = 0; k < s.n_dihedrals; ++k) {
      const uint32_t* d = s.dihedrals + 5 * (size_t)k;
      const uint32_t idx = static_cast<uint32_t>(h_dihedrals.size());
      h_dihedrals.push_back(make_uint4(base + d[0] - 1, base + d[1] - 1, base + d[2] - 1,
                                       base + d[3] - 1));
      h_dih_type.push_back(rp[r].dihedral_type_base + d[4] - 1);
      for (uint32_t m = 0; m < 4; ++m) member[base + d[m] - 1].push_back(term_pack(kTermDihedral, m, idx));
    }
  }
  if (h_bonds.size() >= (1u << 28) || h_angles.size() >= (1u << 28) ||
      h_dihedrals.size() >= (1u << 28)) {
    throw OverflowError("bonded term count exceeds 2^28.");
  }
  std::vector<uint32_t> term_off(T + 1, 0), term;
  for (uint32_t t = 0; t < T; ++t) {
    term_off[t + 1] = term_off[t] + static_cast<uint32_t>(member[t].size());
  }
  term.reserve(term_off[T]);
  for (uint32_t t = 0; t < T; ++t) term.insert(term.end(), member[t].begin(), member[t].end());
  // The membership entry of every (term, member), for k_bonded_terms.
  const size_t nb_all = h_bonds.size(), na_all = h_angles.size(), nd_all = h_dihedrals.size();
  std::vector<uint32_t> term_mem(2 * nb_all + 3 * na_all + 4 * nd_all, 0);
  for (uint32_t e = 0; e < term.size(); ++e) {
    const uint32_t m = term[e];
    const uint32_t kind = m >> 30, role = (m >> 28) & 3u, idx = m & 0x0fffffffu;
    const size_t at = kind == kTermBond    ? 2 * static_cast<size_t>(idx) + role
                      : kind == kTermAngle ? 2 * nb_all + 3 * static_cast<size_t>(idx) + role
                                           : 2 * nb_all + 3 * na_all + 4 * static_cast<size_t>(idx) + role;
    term_mem[at] = e;
  }

  // ---- LJ tables ----
  std::vector<LjCoeff> h_lj(lj_entries);
  for (uint32_t r = 0; r < n; ++r) {
    const beads_forcefield_desc& f = ffs[r];
    const float rc = static_cast<float>(f.lj_cutoff);
    for (int i = 0; i < f.n_types; ++i) {
      for (int j = 0; j < f.n_types; ++j) {
        const float eps = static_cast<float>(f.lj_epsilon[i * f.n_types + j]);
        const float sig = static_cast<float>(f.lj_sigma[i * f.n_types + j]);
        LjCoeff c;
        c.sigma2 = sig * sig;
        c.eps4 = 4.0f * eps;
        c.eps24 = 6.0f * c.eps4;
        c.shift = 0.0f;
        if (f.lj_shift) {
          const float sr2 = c.sigma2 / (rc * rc);
          const float sr6 = sr2 * sr2 * sr2;
          c.shift = c.eps4 * (sr6 * sr6 - sr6);
        }
        h_lj[rp[r].lj_offset + i * f.n_types + j] = c;
      }
    }
  }

  // ---- device allocation ----
  DeviceView& v = v_;
  v.n_replicas = n;
  v.n_slots = S;
  v.n_blocks = S / kBlock;
  v.total_cells = C;
  v.nbr_stride = stride;
  v.excl_cap = static_cast<uint32_t>(excl_cap);
  v.has_bonded = any_bonded ? 1 : 0;
  v.list_by_q = staged_ ? 1 : 0;
  v.stage_cap = stage_cap_;
  v.pos = dalloc<float4>(S + 1);
  v.vel = dalloc<float4>(S);
  v.force = dalloc<float4>(S);
  v.img = dalloc<int4>(S);
  v.tag = dalloc<uint32_t>(S);
  v.mol = dalloc<uint32_t>(S);
  v.ref_pos = dalloc<float4>(S);
  v.ref_img = dalloc<int4>(S);
  v.cross = dalloc<uint32_t>(S);
  v.work_start = dalloc<uint32_t>(n + 1);
  v.chain_block_start = dalloc<uint32_t>(n + 1);
  v.chain_block_list = n > 1 ? 1u : 0u;
  {
    std::vector<uint32_t> chunk_replica, chunk_first(n + 1);
    for (uint32_t r = 0; r < n; ++r) {
      chunk_first[r] = static_cast<uint32_t>(chunk_replica.size());
      const uint32_t chunks = std::max<uint32_t>(1, (rp[r].n_cells + kScanChunk - 1) / kScanChunk);
      chunk_replica.insert(chunk_replica.end(), chunks, r);
    }
    chunk_first[n] = static_cast<uint32_t>(chunk_replica.size());
    uint32_t* d_cr = dalloc<uint32_t>(chunk_replica.size());
    uint32_t* d_cf = dalloc<uint32_t>(n + 1);
    h2d(d_cr, chunk_replica.data(), chunk_replica.size() * 4, "h2d");
    h2d(d_cf, chunk_first.data(), (n + 1) * 4ull, "h2d");
    v.scan_chunk_replica = d_cr;
    v.scan_chunk_first = d_cf;
    v.scan_chunk_sum = dalloc<uint32_t>(chunk_replica.size());
    v.n_scan_chunks = static_cast<uint32_t>(chunk_replica.size());
  }
  v.pos2 = dalloc<float4>(S);
  v.vel2 = dalloc<float4>(S);
  v.img2 = dalloc<int4>(S);
  v.tag2 = dalloc<uint32_t>(S);
  v.mol2 = dalloc<uint32_t>(S);
  v.cell2 = dalloc<uint32_t>(S);
  v.cell_of_slot = dalloc<uint32_t>(S);
  v.cell_count = dalloc<uint32_t>(C);
  v.cell_cursor = dalloc<uint32_t>(C);
  v.cell_start = dalloc<uint32_t>(static_cast<size_t>(C) + n);
  v.cell_atoms = dalloc<uint32_t>(S);
  v.nbr_count = dalloc<uint32_t>(S);
  v.nbr = dalloc<uint32_t>(list_entries);
  v.slot_of_tag = dalloc<uint32_t>(T);
  v.excl_slot = dalloc<uint32_t>(static_cast<size_t>(S) * std::max(1, excl_cap));
  uint32_t* d_excl_off = dalloc<uint32_t>(T + 1);
  uint32_t* d_excl_tag = dalloc<uint32_t>(excl_tag.size());
  uint32_t* d_term_off = dalloc<uint32_t>(T + 1);
  uint32_t* d_term = dalloc<uint32_t>(term.size());
  uint32_t* d_term_mem = dalloc<uint32_t>(term_mem.size());
  v.bonded_contrib = dalloc<float4>(term.size());
  v.bonded_vir = dalloc<float>(term.size());
  uint4* d_bonds = dalloc<uint4>(h_bonds.size());
  uint4* d_angles = dalloc<uint4>(h_angles.size());
  uint4* d_dihedrals = dalloc<uint4>(h_dihedrals.size());
  uint32_t* d_dih_type = dalloc<uint32_t>(h_dih_type.size());
  BondCoeff* d_bc = dalloc<BondCoeff>(h_bc.size());
  AngleCoeff* d_ac = dalloc<AngleCoeff>(h_ac.size());
  DihedralCoeff* d_dc = dalloc<DihedralCoeff>(h_dc.size());
  ReplicaParams* d_rp = dalloc<ReplicaParams>(n);
  v.rs = dalloc<ReplicaState>(n);
  v.obs = dalloc<ReplicaObs>(n);
  uint32_t* d_block_replica = dalloc<uint32_t>(block_replica.size());
  std::vector<uint32_t> cell_replica(C);
  for (uint32_t r = 0; r < n; ++r) {
    std::fill(cell_replica.begin() + rp[r].cell_begin,
              cell_replica.begin() + rp[r].cell_begin + rp[r].n_cells, r);
  }
  uint32_t* d_cell_replica = dalloc<uint32_t>(C);
  v.chain_launches = dalloc<unsigned long long>(1);
  v.ke_part = dalloc<long long>(2ull * n * kKeBuckets);  // zeroed; emptied by every finish
  cuda_check(cudaMemsetAsync(v.chain_launches, 0, sizeof(unsigned long long), stream_), "memset");
  LjCoeff* d_lj = dalloc<LjCoeff>(h_lj.size());

  auto up = [&](void* dst, const void* src, size_t bytes) {
    if (bytes) cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_), "upload");
  };
  up(v.pos, h_pos.data(), (S + 1) * sizeof(float4));
  up(v.vel, h_vel.data(), S * sizeof(float4));
  up(v.img, h_img.data(), S * sizeof(int4));
  up(v.tag, h_tag.data(), S * sizeof(uint32_t));
  up(v.mol, h_mol.data(), S * sizeof(uint32_t));
  up(v.slot_of_tag, slot_of_tag.data(), T * sizeof(uint32_t));
  up(d_excl_off, excl_off.data(), excl_off.size() * sizeof(uint32_t));
  up(d_excl_tag, excl_tag.data(), excl_tag.size() * sizeof(uint32_t));
  up(d_term_off, term_off.data(), term_off.size() * sizeof(uint32_t));
  up(d_term, term.data(), term.size() * sizeof(uint32_t));
  up(d_term_mem, term_mem.data(), term_mem.size() * sizeof(uint32_t));
  up(d_bonds, h_bonds.data(), h_bonds.size() * sizeof(uint4));
  up(d_angles, h_angles.data(), h_angles.size() * sizeof(uint4));
  up(d_dihedrals, h_dihedrals.data(), h_dihedrals.size() * sizeof(uint4));
  up(d_dih_type, h_dih_type.data(), h_dih_type.size() * sizeof(uint32_t));
  up(d_bc, h_bc.data(), h_bc.size() * sizeof(BondCoeff));
  up(d_ac, h_ac.data(), h_ac.size() * sizeof(AngleCoeff));
  up(d_dc, h_dc.data(), h_dc.size() * sizeof(DihedralCoeff));
  up(d_rp, rp.data(), n * sizeof(ReplicaParams));
  up(d_block_replica, block_replica.data(), block_replica.size() * sizeof(uint32_t));
  up(d_cell_replica, cell_replica.data(), C * sizeof(uint32_t));
  up(d_lj, h_lj.data(), h_lj.size() * sizeof(LjCoeff));
  std::vector<ReplicaState> rs(n);
  std::memset(rs.data(), 0, n * sizeof(ReplicaState));
  for (auto& x : rs) x.lambda = 1.0;
  up(v.rs, rs.data(), n * sizeof(ReplicaState));
  v.excl_off = d_excl_off;
  v.excl_tag = d_excl_tag;
  v.term_off = d_term_off;
  v.term = d_term;
  v.bonds = d_bonds;
  v.angles = d_angles;
  v.dihedrals = d_dihedrals;
  v.dihedral_type = d_dih_type;
  v.term_mem = d_term_mem;
  v.n_bond_terms = static_cast<uint32_t>(nb_all);
  v.n_angle_terms = static_cast<uint32_t>(na_all);
  v.n_dihedral_terms = static_cast<uint32_t>(nd_all);
  v.bond_coeff = d_bc;
  v.angle_coeff = d_ac;
  v.dihedral_coeff = d_dc;
  v.rp = d_rp;
  v.block_replica = d_block_replica;
  v.cell_replica = d_cell_replica;
  v.lj = d_lj;

  cuda_check(cudaMallocHost(&h_obs_, n * sizeof(ReplicaObs)), "cudaMallocHost");
  cuda_check(cudaMallocHost(&h_state_, n * sizeof(ReplicaState)), "cudaMallocHost");
  cuda_check(cudaMallocHost(&h_chunk_status_, kStatusRing * n * sizeof(unsigned)),
             "cudaMallocHost");
  for (cudaEvent_t& e : chunk_event_) {
    cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event create");
  }

  launch_.v = v;
  launch_.stream = stream_;
  launch_.max_cells_per_replica = max_cells;
  launch_.lj_tpa = 1;
  launch_.lj_unroll = 8;
  launch_.lj_no_l1 = 0;
  launch_.fuse_post = 0;
  {
    int max_nt = 0;
    for (uint32_t r = 0; r < n; ++r) max_nt = std::max(max_nt, ffs[r].n_types);
    launch_.lj_types = max_nt;
  }
  launch_.max_atoms_per_replica = max_atoms;
  launch_.excl_cap = excl_cap;
  launch_.need_kinetic = any_thermostat ? 1 : 0;
  launch_.any_dense = any_dense_ ? 1 : 0;
  launch_.any_sparse = any_sparse_ ? 1 : 0;
  {
    // One wave of 128-thread blocks (16 per SM) for the chain's per-slot
    // kernels when they walk the block list.
    int device = 0, sms = 0;
    cuda_check(cudaGetDevice(&device), "device");
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
    launch_.chain_grid = std::max<uint32_t>(1u, std::min<uint32_t>(v.n_blocks, 16u * sms));
  }
  if (staged_) prepare_staged_kernels(static_cast<size_t>(stage_cap_ + 1) * sizeof(float4));
  // Initial slot-space exclusion rows (slot order = input order).
  launch_project_exclusions(launch_, true);
  cuda_check(cudaStreamSynchronize(stream_), "setup");
  host_row_tag_ = std::move(h_tag);
}

void Engine::sync() { cuda_check(cudaStreamSynchronize(stream_), "stream synchronize"); }

void Engine::h2d(void* dst, const void* src, size_t bytes, const char* what) {
  cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_), what);
  sync();
}

void Engine::d2h(void* dst, const void* src, size_t bytes, const char* what) {
  cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream_), what);
  sync();
}

void Engine::check_status() {
  sync();
  d2h(h_state_, v_.rs, rep_.size() * sizeof(ReplicaState), "status download");
  for (uint32_t r = 0; r < rep_.size(); ++r) {
    const unsigned s = h_state_[r].status;
    if (s & kStatusNeighborOverflow) {
      const ReplicaHost& h = rep_[r];
      std::ostringstream m;
      m << "NeighborList overflow"
        << "\npath=" << path_name(h.plan.path) << "\nn_particles=" << h.n_atoms
        << "\nmax_neighbors=" << h.max_neighbors << "\nforce_cutoff=" << h.plan.force_cutoff
        << "\ncutoff_buffer=" << h.plan.cutoff_buffer
        << "\nsearch_cutoff=" << h.plan.search_cutoff
        << ". Increase max_neighbors before consuming this neighbor list.";
      if (rep_.size() > 1) m << " (replica " << r << ")";
      throw NeighborOverflow(m.str());
    }
    if (s & kStatusFixedOverflow) {
      throw OverflowError("energy, virial or kinetic energy of a particle is not finite or "
                          "exceeds the fixed-point accumulator range (|value| < 4e18).");
    }
    if (s & kStatusNonFinite) {
      throw NonFinite("non-finite velocity after force evaluation (replica " +
                      std::to_string(r) + ").");
    }
  }
}

void Engine::eval() {
  TraceRange trace("beads.eval");
  launch_apply_lambda(launch_);
  launch_rebuild(launch_, true);
  launch_forces(launch_, true, false);
  launch_post(launch_, false, true);
  check_status();
  initialized_ = true;
}

void Engine::record_step(bool observables) {
  launch_pre(launch_, kPreVerlet);
  launch_rebuild(launch_, false);
  launch_forces(launch_, observables, false, true);
}

// One step inside a stream capture, with the rebuild chain as the body of an
// IF conditional node that the pre kernel switches on (CUDA 12.4+ graphs).
// Steps without a rebuild then launch only pre and the force kernel(s), the
// last of which also does the second half-kick.
void Engine::record_step_conditional(bool observables) {
  cudaStreamCaptureStatus status;
  cudaGraph_t graph = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t n_deps = 0;
  cuda_check(cudaStreamGetCaptureInfo(stream_, &status, nullptr, &graph, &deps, &n_deps),
             "capture info");
  cudaGraphConditionalHandle handle;
  cuda_check(cudaGraphConditionalHandleCreate(&handle, graph, 0, cudaGraphCondAssignDefault),
             "conditional handle");
  launch_pre(launch_, kPreVerlet, handle, true);
  cuda_check(cudaStreamGetCaptureInfo(stream_, &status, nullptr, &graph, &deps, &n_deps),
             "capture info");
  cudaGraphNodeParams params = {};
  params.type = cudaGraphNodeTypeConditional;
  params.conditional.handle = handle;
  params.conditional.type = cudaGraphCondTypeIf;
  params.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  cuda_check(cudaGraphAddNode(&node, graph, deps, n_deps, &params), "conditional node");
  cudaGraph_t body = params.conditional.phGraph_out[0];
  cuda_check(cudaStreamUpdateCaptureDependencies(stream_, &node, 1,
                                                 cudaStreamSetCaptureDependencies),
             "capture dependencies");
  if (!side_stream_) {
    cuda_check(cudaStreamCreateWithFlags(&side_stream_, cudaStreamNonBlocking), "stream create");
  }
  StepLaunch side = launch_;
  side.stream = side_stream_;
  cuda_check(cudaStreamBeginCaptureToGraph(side_stream_, body, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal),
             "body capture");
  try {
    launch_rebuild(side, false);
  } catch (...) {
    cudaGraph_t discard = nullptr;
    cudaStreamEndCapture(side_stream_, &discard);
    throw;
  }
  cuda_check(cudaStreamEndCapture(side_stream_, &body), "body capture end");
  last_chain_body_ = body;
  launch_forces(launch_, observables, false, true);
}

cudaGraphExec_t Engine::graph_for(uint32_t steps, bool obs_last) {
  const auto key = std::make_pair(steps, obs_last);
  auto it = graphs_.find(key);
  if (it != graphs_.end()) return it->second.second;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  for (int attempt = 0; attempt < 2; ++attempt) {
    const bool conditional = use_conditional_;
    cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
      for (uint32_t s = 0; s < steps; ++s) {
        const bool obs = obs_last && s + 1 == steps;
        if (conditional) {
          record_step_conditional(obs);
        } else {
          record_step(obs);
        }
      }
      cuda_check(cudaStreamEndCapture(stream_, &graph), "end capture");
      cuda_check(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
      break;
    } catch (const CudaError&) {
      cudaGraph_t discard = nullptr;
      cudaStreamEndCapture(stream_, &discard);
      if (discard) cudaGraphDestroy(discard);
      if (graph) cudaGraphDestroy(graph);
      graph = nullptr;
      cudaGetLastError();
      // Conditional nodes refused (older driver): capture the same step with
      // the rebuild kernels returning early instead.
      if (!conditional) throw;
      use_conditional_ = false;
    } catch (...) {
      cudaGraph_t discard = nullptr;
      cudaStreamEndCapture(stream_, &discard);
      if (discard) cudaGraphDestroy(discard);
      throw;
    }
  }
  graphs_[key] = std::make_pair(graph, exec);
  return exec;
}

void Engine::launch_counts(uint32_t& per_step, uint32_t& per_chain) {
  // The cached one-step graph settles whether this driver takes conditional
  // nodes (graph_for falls back to recording the chain in every step).
  if (use_graphs_) graph_for(1, false);
  const bool conditional = use_graphs_ && use_conditional_;
  sync();
  cudaGraph_t graph = nullptr;
  cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
  try {
    if (conditional) {
      record_step_conditional(false);
    } else {
      record_step(false);
    }
  } catch (...) {
    cudaGraph_t discard = nullptr;
    cudaStreamEndCapture(stream_, &discard);
    if (discard) cudaGraphDestroy(discard);
    throw;
  }
  cuda_check(cudaStreamEndCapture(stream_, &graph), "end capture");
  // Every node a step records is a kernel launch, except the conditional
  // node that holds the rebuild chain (whose body holds only kernels).  The
  // graphs are only queried once the capture has ended.
  size_t top = 0, body = 0;
  cudaError_t e = cudaGraphGetNodes(graph, nullptr, &top);
  if (e == cudaSuccess && conditional) e = cudaGraphGetNodes(last_chain_body_, nullptr, &body);
  last_chain_body_ = nullptr;
  cudaGraphDestroy(graph);
  cuda_check(e, "graph nodes");
  per_step = static_cast<uint32_t>(conditional ? top - 1 : top);
  per_chain = static_cast<uint32_t>(body);
}

void Engine::launch_chunk(uint32_t steps, bool obs_last) {
  if (use_graphs_) {
    cuda_check(cudaGraphLaunch(graph_for(steps, obs_last), stream_), "graph launch");
  } else {
    for (uint32_t s = 0; s < steps; ++s) record_step(obs_last && s + 1 == steps);
  }
}

bool Engine::run(uint64_t steps, uint64_t obs_every, const std::function<bool()>* poll,
                 uint64_t poll_every) {
  TraceRange trace("beads.run");
  if (!initialized_) eval();
  if (!tuned_ && !tuning_fixed_ && steps > 0) autotune();
  const uint32_t n = n_replicas();
  bool last_obs = false;
  uint64_t remaining = steps;
  uint64_t chunks = 0;
  uint64_t last_poll = step_;
  // Status words of a finished chunk: any bit set means the step that set it
  // failed; check_status() (full download, reference message) then throws.
  auto chunk_failed = [&](uint64_t k) {
    const unsigned* w = h_chunk_status_ + (k % kStatusRing) * n;
    for (uint32_t r = 0; r < n; ++r) {
      if (w[r] != 0u) return true;
    }
    return false;
  };
  while (remaining > 0) {
    uint64_t chunk = std::min<uint64_t>(remaining, kChunkMax);
    bool obs = false;
    if (obs_every > 0) {
      const uint64_t next = (step_ / obs_every + 1) * obs_every;
      if (next - step_ <= chunk) {
        chunk = next - step_;
        obs = true;
      }
    }
    // Chunks are powers of two, so a run of any length replays at most
    // log2(kChunkMax) + 1 distinct captured graphs (instantiated once each).
    uint64_t pow2 = 1;
    while (pow2 * 2 <= chunk) pow2 *= 2;
    if (pow2 != chunk) {
      chunk = pow2;
      obs = false;
    }
    launch_chunk(static_cast<uint32_t>(chunk), obs);
    // This chunk's status words, gathered from the replica states (one
    // strided copy), land in its slot of the pinned ring.
    const uint64_t k = chunks++;
    cuda_check(cudaMemcpy2DAsync(h_chunk_status_ + (k % kStatusRing) * n, sizeof(unsigned),
                                 &v_.rs->status,
                                 sizeof(ReplicaState), sizeof(unsigned), n,
                                 cudaMemcpyDeviceToHost, stream_),
               "status copy");
    cuda_check(cudaEventRecord(chunk_event_[k % kStatusRing], stream_), "event record");
    step_ += chunk;
    remaining -= chunk;
    last_obs = obs;
    // Check the chunk two before this one: the GPU still holds the last two
    // chunks while the host waits, so a host stall of up to a chunk's length
    // leaves it no idle gap.  A failure is raised at most two chunks after
    // the chunk that set it (every chunk left is checked at the end).
    constexpr uint64_t kLag = kStatusRing - 1;
    if (k >= kLag) {
      cuda_check(cudaEventSynchronize(chunk_event_[(k - kLag) % kStatusRing]), "status wait");
      if (chunk_failed(k - kLag)) check_status();
    }
    if (poll != nullptr && remaining > 0 && step_ - last_poll >= poll_every) {
      last_poll = step_;
      if ((*poll)()) {
        sync();
        check_status();
        throw std::runtime_error("interrupted");  // BEADS_ERR_INTERRUPTED
      }
    }
  }
  check_status();
  return last_obs;
}

void Engine::minimize(uint32_t iterations, float dmax, float fref) {
  TraceRange trace("beads.minimize");
  StepLaunch l = launch_;
  l.sd_dmax = dmax;
  l.sd_fref = fref;
  launch_rebuild(l, true);
  for (uint32_t it = 0; it < iterations; ++it) {
    launch_forces(l, false, true);
    launch_pre(l, kPreDescent);
    launch_rebuild(l, false);
  }
  sync();
  // The descent is set-up work: reset counters so a following run starts
  // like a fresh one.
  check_status();
  for (uint32_t r = 0; r < rep_.size(); ++r) {
    h_state_[r].builds = 0;
    h_state_[r].dangerous = 0;
    h_state_[r].checks_since_build = 0;
    h_state_[r].need_rebuild = 0;
    h_state_[r].reorder_now = 0;
    h_state_[r].step = 0;
    h_state_[r].lambda = 1.0;
  }
  h2d(v_.rs, h_state_, rep_.size() * sizeof(ReplicaState), "state reset");
  initialized_ = false;
  step_ = 0;
}

void Engine::flush_lambda() { launch_apply_lambda(launch_); }

double Engine::profile(int stage, uint32_t reps) {
  if (!initialized_) eval();
  if (reps == 0) reps = 1;
  cudaEvent_t start = nullptr, stop = nullptr;
  cuda_check(cudaEventCreate(&start), "event create");
  cuda_check(cudaEventCreate(&stop), "event create");
  float ms = 0.f;
  std::vector<ReplicaState> saved;
  if (stage == 3) {
    // The kick variant changes velocities and the per-replica step state:
    // keep copies and put them back after timing.
    saved.resize(rep_.size());
    sync();
    d2h(saved.data(), v_.rs, saved.size() * sizeof(ReplicaState), "state save");
    cuda_check(cudaMemcpyAsync(v_.vel2, v_.vel, v_.n_slots * sizeof(float4),
                               cudaMemcpyDeviceToDevice, stream_), "velocity save");
  }
  try {
    sync();
    cuda_check(cudaEventRecord(start, stream_), "event record");
    for (uint32_t k = 0; k < reps; ++k) {
      if (stage == 0) {
        launch_forces(launch_, false, false);
      } else if (stage == 3) {
        launch_forces(launch_, false, false, true);
      } else if (stage == 1) {
        launch_chunk(1, false);
        step_ += 1;
      } else if (stage == 2) {
        launch_rebuild(launch_, true);
      } else if (stage == 4) {
        launch_forces(launch_, false, false, false, kForcePair);
      } else if (stage == 5) {
        launch_forces(launch_, false, false, false, kForceBonded);
      } else {
        throw InvalidArgument("unknown profile stage");
      }
    }
    cuda_check(cudaEventRecord(stop, stream_), "event record");
    cuda_check(cudaEventSynchronize(stop), "event sync");
    cuda_check(cudaEventElapsedTime(&ms, start, stop), "event elapsed");
  } catch (...) {
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    throw;
  }
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  // The pair-only and bonded-only stages leave partial (or repeatedly added)
  // forces: one full evaluation restores them.
  if (stage == 4 || stage == 5) launch_forces(launch_, false, false);
  if (stage == 3) {
    cuda_check(cudaMemcpyAsync(v_.vel, v_.vel2, v_.n_slots * sizeof(float4),
                               cudaMemcpyDeviceToDevice, stream_), "velocity restore");
    cuda_check(cudaMemcpyAsync(v_.rs, saved.data(), saved.size() * sizeof(ReplicaState),
                               cudaMemcpyHostToDevice, stream_), "state restore");
    sync();
  }
  check_status();
  return static_cast<double>(ms) / reps;
}

void Engine::counters(uint32_t replica, uint64_t out[4]) {
  sync();
  ReplicaState st;
  d2h(&st, v_.rs + replica, sizeof(ReplicaState), "counters download");
  out[0] = st.step;
  out[1] = st.builds;
  out[2] = st.dangerous;
  d2h(&out[3], v_.chain_launches, sizeof(unsigned long long), "counters download");
}

void Engine::list_stats(uint64_t* total, uint32_t* max_count) {
  sync();
  std::vector<uint32_t> cnt(v_.n_slots);
  d2h(cnt.data(), v_.nbr_count, cnt.size() * 4ull, "d2h");
  uint64_t t = 0;
  uint32_t m = 0;
  for (uint32_t c : cnt) {
    t += c;
    m = std::max(m, c);
  }
  if (total) *total = t;
  if (max_count) *max_count = m;
}

void Engine::observables(std::vector<beads_observables>& out) {
  sync();
  d2h(h_obs_, v_.obs, rep_.size() * sizeof(ReplicaObs), "observables download");
  out.resize(rep_.size());
  for (uint32_t r = 0; r < rep_.size(); ++r) {
    const ReplicaObs& o = h_obs_[r];
    const ReplicaHost& h = rep_[r];
    beads_observables& b = out[r];
    b.step = o.step;
    b.pair_pe = o.pair_pe;
    b.bond_pe = o.bond_pe;
    b.angle_pe = o.angle_pe;
    b.dihedral_pe = o.dihedral_pe;
    b.pe = o.pair_pe + o.bond_pe + o.angle_pe + o.dihedral_pe;
    b.ke = o.lambda * o.lambda * o.ke_pre;
    b.virial = o.virial;
    const double kb = h.units == BEADS_UNITS_NM_KJMOL ? kKbNmKjMol : 1.0;
    const double ps = h.units == BEADS_UNITS_NM_KJMOL ? kPressNmKjMol : 1.0;
    const double dof = std::max(0.0, 3.0 * h.n_atoms - 3.0);
    b.temp = (dof > 0.0) ? 2.0 * b.ke / (dof * kb) : 0.0;
    const double vol = static_cast<double>(h.box_hi[0] - h.box_lo[0]) *
                       static_cast<double>(h.box_hi[1] - h.box_lo[1]) *
                       static_cast<double>(h.box_hi[2] - h.box_lo[2]);
    b.press = vol > 0.0 ? ps * (2.0 * b.ke + b.virial) / (3.0 * vol) : 0.0;
    b.neighbor_build_count = o.builds;
    b.dangerous_rebuild_count = o.dangerous;
  }
}

void Engine::slot_view(uint32_t r, SlotView& out) {
  const ReplicaHost& h = rep_.at(r);
  flush_lambda();
  sync();
  const size_t n = h.n_atoms;
  out.pos.resize(n);
  out.vel.resize(n);
  out.force.resize(n);
  out.img.resize(n);
  out.tag.resize(n);
  out.mol.resize(n);
  const size_t b = h.atom_begin;
  d2h(out.pos.data(), v_.pos + b, n * sizeof(float4), "d2h");
  d2h(out.vel.data(), v_.vel + b, n * sizeof(float4), "d2h");
  d2h(out.force.data(), v_.force + b, n * sizeof(float4), "d2h");
  d2h(out.img.data(), v_.img + b, n * sizeof(int4), "d2h");
  d2h(out.tag.data(), v_.tag + b, n * sizeof(uint32_t), "d2h");
  d2h(out.mol.data(), v_.mol + b, n * sizeof(uint32_t), "d2h");
  for (auto& t : out.tag) t = t - h.tag_base + 1;  // 1-based local tags
}

void Engine::state(uint32_t r, float* pos, float* vel, float* force, int32_t* img,
                   uint32_t*, int32_t*) {
  SlotView sv;
  slot_view(r, sv);
  for (size_t k = 0; k < sv.tag.size(); ++k) {
    const size_t t = sv.tag[k] - 1;
    if (pos) {
      pos[3 * t] = sv.pos[k].x;
      pos[3 * t + 1] = sv.pos[k].y;
      pos[3 * t + 2] = sv.pos[k].z;
    }
    if (vel) {
      vel[3 * t] = sv.vel[k].x;
      vel[3 * t + 1] = sv.vel[k].y;
      vel[3 * t + 2] = sv.vel[k].z;
    }
    if (force) {
      force[3 * t] = sv.force[k].x;
      force[3 * t + 1] = sv.force[k].y;
      force[3 * t + 2] = sv.force[k].z;
    }
    if (img) {
      img[3 * t] = sv.img[k].x;
      img[3 * t + 1] = sv.img[k].y;
      img[3 * t + 2] = sv.img[k].z;
    }
  }
}

void Engine::set_state(uint32_t r, const float* pos, const float* vel) {
  const ReplicaHost& h = rep_.at(r);
  if (pos) {
    for (uint64_t k = 0; k < 3ull * h.n_atoms; ++k) {
      const int a = static_cast<int>(k % 3);
      if (!(pos[k] >= h.box_lo[a] && pos[k] < h.box_hi[a])) {
        throw InvalidArgument("positions must be inside box_bound");
      }
    }
  }
  if (!d_xfer_pos_) {
    d_xfer_pos_ = dalloc<float>(3 * n_tags_);
    d_xfer_vel_ = dalloc<float>(3 * n_tags_);
  }
  flush_lambda();
  const size_t off = 3ull * h.tag_base;
  const size_t bytes = 3ull * h.n_atoms * sizeof(float);
  // Stage this replica's rows and scatter only them: the kernel walks all
  // tags, so the other replicas' rows are first refreshed from the device.
  launch_gather_state(launch_, d_xfer_pos_, d_xfer_vel_, static_cast<uint32_t>(n_tags_));
  if (pos) cuda_check(cudaMemcpyAsync(d_xfer_pos_ + off, pos, bytes, cudaMemcpyHostToDevice, stream_), "h2d");
  if (vel) cuda_check(cudaMemcpyAsync(d_xfer_vel_ + off, vel, bytes, cudaMemcpyHostToDevice, stream_), "h2d");
  launch_scatter_state(launch_, d_xfer_pos_, d_xfer_vel_, static_cast<uint32_t>(n_tags_));
  sync();
  initialized_ = false;
}

void Engine::upload_all(const float* pos, const float* vel) {
  if (!d_xfer_pos_) {
    d_xfer_pos_ = dalloc<float>(3 * n_tags_);
    d_xfer_vel_ = dalloc<float>(3 * n_tags_);
  }
  const size_t bytes = 3ull * n_tags_ * sizeof(float);
  flush_lambda();
  if (pos) cuda_check(cudaMemcpyAsync(d_xfer_pos_, pos, bytes, cudaMemcpyHostToDevice, stream_), "h2d");
  if (vel) cuda_check(cudaMemcpyAsync(d_xfer_vel_, vel, bytes, cudaMemcpyHostToDevice, stream_), "h2d");
  launch_scatter_state(launch_, pos ? d_xfer_pos_ : nullptr, vel ? d_xfer_vel_ : nullptr,
                       static_cast<uint32_t>(n_tags_));
  // From pinned host memory the copies are asynchronous: the caller may reuse
  // its buffers as soon as this returns.
  sync();
  initialized_ = false;
}

void Engine::download_all(float* pos, float* vel) {
  if (!d_xfer_pos_) {
    d_xfer_pos_ = dalloc<float>(3 * n_tags_);
    d_xfer_vel_ = dalloc<float>(3 * n_tags_);
  }
  const size_t bytes = 3ull * n_tags_ * sizeof(float);
  flush_lambda();
  launch_gather_state(launch_, d_xfer_pos_, d_xfer_vel_, static_cast<uint32_t>(n_tags_));
  if (pos) cuda_check(cudaMemcpyAsync(pos, d_xfer_pos_, bytes, cudaMemcpyDeviceToHost, stream_), "d2h");
  if (vel) cuda_check(cudaMemcpyAsync(vel, d_xfer_vel_, bytes, cudaMemcpyDeviceToHost, stream_), "d2h");
  sync();
}

void Engine::debug_cells(uint32_t r, uint32_t* cell_by_tag) {
  const ReplicaHost& h = rep_.at(r);
  sync();
  std::vector<uint32_t> cell(h.n_atoms), tag(h.n_atoms);
  d2h(cell.data(), v_.cell_of_slot + h.atom_begin, h.n_atoms * 4, "d2h");
  d2h(tag.data(), v_.tag + h.atom_begin, h.n_atoms * 4, "d2h");
  std::vector<ReplicaParams> rp(1);
  d2h(rp.data(), v_.rp + r, sizeof(ReplicaParams), "d2h");
  for (uint32_t k = 0; k < h.n_atoms; ++k) {
    cell_by_tag[tag[k] - h.tag_base] = cell[k] - rp[0].cell_begin;
  }
}

void Engine::set_list_staged(bool staged) {
  const bool want = staged && stage_cap_ > 0;
  layout_fixed_ = true;
  if ((v_.list_by_q != 0) == want) return;
  clear_graphs();
  v_.list_by_q = want ? 1 : 0;
  launch_.v = v_;
  if (initialized_) relayout_list();
}

// Rebuilds the current list in the current layout from the positions of the
// last build (ref_pos), without counting a build or reordering: the same
// cells, the same candidates in the same order, so the same list.  The
// displacement reference (images and crossing counts since that build) and
// the positions are restored afterwards, so the dynamics continue bit for
// bit as they would have without the change.
void Engine::relayout_list() {
  const size_t S = v_.n_slots;
  // Save buffers kept for the context's life (allocated at the first call):
  // a layout change, the autotuner's included, then costs no allocation.
  if (!relayout_pos_) {
    relayout_pos_ = dalloc<float4>(S);
    relayout_img_ = dalloc<int4>(S);
    relayout_cross_ = dalloc<uint32_t>(S);
  }
  auto d2d = [&](void* dst, const void* src, size_t bytes) {
    cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream_), "copy");
  };
  d2d(relayout_pos_, v_.pos, S * sizeof(float4));
  d2d(relayout_img_, v_.ref_img, S * sizeof(int4));
  d2d(relayout_cross_, v_.cross, S * sizeof(uint32_t));
  d2d(v_.pos, v_.ref_pos, S * sizeof(float4));
  std::vector<ReplicaState> saved(rep_.size());
  sync();
  d2h(saved.data(), v_.rs, saved.size() * sizeof(ReplicaState), "state save");
  launch_rebuild(launch_, true, false);
  d2d(v_.pos, relayout_pos_, S * sizeof(float4));
  d2d(v_.ref_img, relayout_img_, S * sizeof(int4));
  d2d(v_.cross, relayout_cross_, S * sizeof(uint32_t));
  cuda_check(cudaMemcpyAsync(v_.rs, saved.data(), saved.size() * sizeof(ReplicaState),
                             cudaMemcpyHostToDevice, stream_), "state restore");
  sync();
}

void Engine::debug_neighbors(uint32_t r, uint32_t cap, uint32_t* counts, uint32_t* partners) {
  if (v_.list_by_q) {
    debug_neighbors_staged(r, cap, counts, partners);
    return;
  }
  const ReplicaHost& h = rep_.at(r);
  sync();
  const uint32_t S = v_.n_slots;
  std::vector<uint32_t> cnt(S), tag(S);
  d2h(cnt.data(), v_.nbr_count, S * 4ull, "d2h");
  d2h(tag.data(), v_.tag, S * 4ull, "d2h");
  // Only the groups of this replica's slots are copied.
  const uint64_t g0 = h.atom_begin / kGroup, g1 = (h.atom_begin + h.n_pad) / kGroup;
  const uint64_t per_group = static_cast<uint64_t>(v_.nbr_stride) * kGroup;
  std::vector<uint32_t> list((g1 - g0) * per_group);
  d2h(list.data(), v_.nbr + g0 * per_group, list.size() * 4ull, "d2h");
  for (uint32_t k = 0; k < h.n_atoms; ++k) {
    const uint32_t slot = h.atom_begin + k;
    const uint32_t t = tag[slot] - h.tag_base;  // 0-based local
    const uint32_t c = cnt[slot];
    counts[t] = c;
    for (uint32_t q = 0; q < c && q < cap; ++q) {
      const uint64_t at = nbr_index(slot, q, v_.nbr_stride) - g0 * per_group;
      const uint32_t j = list[at];
      partners[static_cast<uint64_t>(t) * cap + q] = tag[j] - h.tag_base + 1;
    }
  }
}

// Staged contexts keep list rows by cell order and stage indices as entries:
// a device pass decodes them into a slot-indexed copy of neighbour slots.
void Engine::debug_neighbors_staged(uint32_t r, uint32_t cap, uint32_t* counts,
                                    uint32_t* partners) {
  const ReplicaHost& h = rep_.at(r);
  sync();
  const uint32_t S = v_.n_slots;
  uint32_t* d_count = nullptr;
  uint32_t* d_list = nullptr;
  cuda_check(cudaMalloc(&d_count, S * 4ull), "cudaMalloc");
  cuda_check(cudaMalloc(&d_list, static_cast<size_t>(S) * cap * 4ull), "cudaMalloc");
  std::vector<uint32_t> cnt(S), tag(S), list(static_cast<size_t>(h.n_atoms) * cap);
  try {
    cuda_check(cudaMemsetAsync(d_count, 0, S * 4ull, stream_), "memset");
    launch_list_to_slots(launch_, cap, d_count, d_list);
    sync();
    d2h(cnt.data(), d_count, S * 4ull, "d2h");
    d2h(list.data(), d_list + static_cast<size_t>(h.atom_begin) * cap, list.size() * 4ull, "d2h");
    d2h(tag.data(), v_.tag, S * 4ull, "d2h");
  } catch (...) {
    cudaFree(d_count);
    cudaFree(d_list);
    throw;
  }
  cudaFree(d_count);
  cudaFree(d_list);
  for (uint32_t k = 0; k < h.n_atoms; ++k) {
    const uint32_t slot = h.atom_begin + k;
    const uint32_t t = tag[slot] - h.tag_base;
    const uint32_t c = cnt[slot];
    counts[t] = c;
    for (uint32_t q = 0; q < c && q < cap; ++q) {
      const uint32_t j = list[static_cast<size_t>(k) * cap + q];
      partners[static_cast<uint64_t>(t) * cap + q] = tag[j] - h.tag_base + 1;
    }
  }
}

}  // namespace bb
