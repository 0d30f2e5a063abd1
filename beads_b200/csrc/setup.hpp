// setup.hpp -- host-side planning: validation, cell grid, exclusions, bonded
// tables.  Plain C++ (no CUDA) so it can be unit-tested on the host.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/beads_b200.h"

namespace bb {

struct InvalidArgument : std::invalid_argument {
  using std::invalid_argument::invalid_argument;
};
struct OverflowError : std::overflow_error {
  using std::overflow_error::overflow_error;
};

enum PathKind : int { kPathDirect = 0, kPathRegular = 1, kPathSmall = 2 };

// Cell grid and neighbour path of one replica.  Follows the reference's
// NeighborPlan (native/src/simulation/neighbor/neighbor_plan.cpp:29-236):
// n_axis = max(1, floor(L / (rc + skin))) evaluated in double on the float
// values, cell = L / n and inv = 1 / cell in float, search cutoff rc + skin in
// float, and rc + skin <= L / 2 required.
struct Plan {
  float force_cutoff = 0.f;
  float cutoff_buffer = 0.f;
  float search_cutoff = 0.f;
  float search_cutoff_sq = 0.f;
  float force_cutoff_sq = 0.f;
  uint32_t nc[3] = {1, 1, 1};
  uint32_t n_cells = 1;
  float cell_size[3] = {0, 0, 0};
  float inv_cell[3] = {0, 0, 0};
  PathKind path = kPathDirect;
};

Plan make_plan(const float box_lo[3], const float box_hi[3], double cutoff,
               double cutoff_buffer);
const char* path_name(PathKind path);

// Validation of one replica's descriptors (messages follow the reference's
// parser/validation wording where a drop-in caller can see them).
void validate_replica(const beads_system_desc& s, const beads_forcefield_desc& f,
                      const beads_neighbor_desc& n, const beads_dynamics_desc& d);

// Pairs within bond-graph distance 1..d, as sorted (tag_i < tag_j) pairs of
// 1-based tags.  Same set as the reference's breadth-first search
// (native/src/system/topology/exclusions.cu:514-598).
std::vector<std::pair<uint32_t, uint32_t>> bond_graph_exclusions(
    uint32_t n_particles, const uint32_t* bonds, uint32_t n_bonds,
    uint32_t distance);

// Row -> tag mapping (1-based tags); NULL tags mean row k has tag k + 1.
std::vector<uint32_t> row_tags(const beads_system_desc& s);

}  // namespace bb
