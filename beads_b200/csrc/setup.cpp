// setup.cpp -- host-side planning and validation.
#include "setup.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <sstream>

namespace bb {
namespace {

void require_finite_positive(double v, const char* what) {
  if (!std::isfinite(v) || v <= 0.0) {
    throw InvalidArgument(std::string(what) + " must be finite and positive.");
  }
}

uint32_t axis_cells(float length, float search_cutoff) {
  const double raw = std::floor(static_cast<double>(length) /
                                static_cast<double>(search_cutoff));
  if (!std::isfinite(raw)) throw InvalidArgument("neighbor cell count must be finite.");
  if (raw < 1.0) return 1u;
  if (raw > static_cast<double>(std::numeric_limits<uint32_t>::max())) {
    throw InvalidArgument("neighbor cell count exceeds index_t range.");
  }
  return static_cast<uint32_t>(raw);
}

}  // namespace

const char* path_name(PathKind path) {
  switch (path) {
    case kPathDirect: return "direct";
    case kPathRegular: return "regular_cell";
    case kPathSmall: return "small_dimension";
  }
  return "unknown";
}

Plan make_plan(const float box_lo[3], const float box_hi[3], double cutoff,
               double cutoff_buffer) {
  Plan p;
  p.force_cutoff = static_cast<float>(cutoff);
  p.cutoff_buffer = static_cast<float>(cutoff_buffer);
  require_finite_positive(p.force_cutoff, "neighbor force_cutoff");
  if (!std::isfinite(p.cutoff_buffer) || p.cutoff_buffer < 0.f) {
    throw InvalidArgument("neighbor cutoff_buffer must be finite and non-negative.");
  }
  p.search_cutoff = p.force_cutoff + p.cutoff_buffer;
  p.search_cutoff_sq = p.search_cutoff * p.search_cutoff;
  p.force_cutoff_sq = p.force_cutoff * p.force_cutoff;
  float len[3];
  for (int a = 0; a < 3; ++a) {
    len[a] = box_hi[a] - box_lo[a];
    require_finite_positive(len[a], "box length");
  }
  const float half_shortest = 0.5f * std::min(len[0], std::min(len[1], len[2]));
  if (p.search_cutoff > half_shortest) {
    throw InvalidArgument(
        "neighbor search_cutoff must not exceed half shortest box length.");
  }
  uint64_t total = 1;
  for (int a = 0; a < 3; ++a) {
    p.nc[a] = axis_cells(len[a], p.search_cutoff);
    total *= p.nc[a];
    if (total > std::numeric_limits<uint32_t>::max()) {
      throw InvalidArgument("neighbor n_cells exceeds index_t range.");
    }
    p.cell_size[a] = len[a] / static_cast<float>(p.nc[a]);
    p.inv_cell[a] = 1.0f / p.cell_size[a];
    if (p.nc[a] >= 3) {
      const float tol = std::max(1.0e-6f, p.search_cutoff * 1.0e-5f);
      if (p.cell_size[a] + tol < p.search_cutoff) {
        throw InvalidArgument("neighbor cell size must be at least neighbor search_cutoff.");
      }
    }
  }
  p.n_cells = static_cast<uint32_t>(total);
  const bool all_small = p.nc[0] < 3 && p.nc[1] < 3 && p.nc[2] < 3;
  const bool all_large = p.nc[0] >= 3 && p.nc[1] >= 3 && p.nc[2] >= 3;
  p.path = all_small ? kPathDirect : (all_large ? kPathRegular : kPathSmall);
  return p;
}

std::vector<uint32_t> row_tags(const beads_system_desc& s) {
  std::vector<uint32_t> tags(s.n_particles);
  for (uint32_t k = 0; k < s.n_particles; ++k) tags[k] = s.tags ? s.tags[k] : k + 1;
  return tags;
}

void validate_replica(const beads_system_desc& s, const beads_forcefield_desc& f,
                      const beads_neighbor_desc& n, const beads_dynamics_desc& d) {
  if (s.n_particles == 0) throw InvalidArgument("system.n_particles must be positive.");
  if (s.units != BEADS_UNITS_REDUCED && s.units != BEADS_UNITS_NM_KJMOL) {
    throw InvalidArgument("system.units must be \"reduced\" or \"nm_kjmol\".");
  }
  if (!s.positions || !s.types) throw InvalidArgument("system positions and types are required.");
  for (int a = 0; a < 3; ++a) {
    if (!std::isfinite(s.box_lo[a]) || !std::isfinite(s.box_hi[a]) ||
        !(s.box_hi[a] > s.box_lo[a])) {
      throw InvalidArgument("system.box_bound upper row must be greater than lower row.");
    }
  }
  const uint32_t n_p = s.n_particles;
  for (uint64_t k = 0; k < 3ull * n_p; ++k) {
    const float x = s.positions[k];
    const int a = static_cast<int>(k % 3);
    if (!std::isfinite(x)) throw InvalidArgument("system.positions must be finite.");
    if (x < s.box_lo[a] || x >= s.box_hi[a]) {
      throw InvalidArgument("system.positions must be inside box_bound.");
    }
    if (s.velocities && !std::isfinite(s.velocities[k])) {
      throw InvalidArgument("system.velocities must be finite.");
    }
  }
  if (f.n_types < 1 || f.n_types > 16) {
    throw InvalidArgument("forcefield supports 1..16 particle types.");
  }
  for (uint32_t k = 0; k < n_p; ++k) {
    if (s.types[k] < 1 || s.types[k] > f.n_types) {
      throw InvalidArgument("system.types must be dense one-based ids covered by pair_coeffs.");
    }
    if (s.masses && !(std::isfinite(s.masses[k]) && s.masses[k] > 0.f)) {
      throw InvalidArgument("system.masses must be finite and positive.");
    }
  }
  if (s.tags) {
    std::vector<uint8_t> seen(n_p + 1, 0);
    for (uint32_t k = 0; k < n_p; ++k) {
      const uint32_t t = s.tags[k];
      if (t < 1 || t > n_p || seen[t]) {
        throw InvalidArgument("system.tags must be a permutation of 1..N.");
      }
      seen[t] = 1;
    }
  }
  if (!f.lj_epsilon || !f.lj_sigma) throw InvalidArgument("pair_coeffs are required.");
  for (int i = 0; i < f.n_types * f.n_types; ++i) {
    if (!(f.lj_epsilon[i] > 0.0) || !(f.lj_sigma[i] > 0.0) ||
        !std::isfinite(f.lj_epsilon[i]) || !std::isfinite(f.lj_sigma[i])) {
      throw InvalidArgument("pair_coeff epsilon and sigma must be finite and positive.");
    }
  }
  if (!(f.lj_cutoff > 0.0) || !std::isfinite(f.lj_cutoff)) {
    throw InvalidArgument("pair_style.params.cutoff must be finite and positive.");
  }
  auto check_terms = [&](const uint32_t* recs, uint32_t count, int width,
                         int n_types, const char* what) {
    if (count == 0) return;
    if (!recs) throw InvalidArgument(std::string(what) + " records are missing.");
    for (uint32_t k = 0; k < count; ++k) {
      for (int m = 0; m < width - 1; ++m) {
        const uint32_t t = recs[(size_t)k * width + m];
        if (t < 1 || t > n_p) {
          throw InvalidArgument(std::string(what) + " reference unknown System tags.");
        }
      }
      const uint32_t ty = recs[(size_t)k * width + width - 1];
      if (ty < 1 || static_cast<int>(ty) > n_types) {
        throw InvalidArgument(std::string(what) + " type has no coefficients.");
      }
    }
  };
  check_terms(s.bonds, s.n_bonds, 3, f.n_bond_types, "bonds");
  check_terms(s.angles, s.n_angles, 4, f.n_angle_types, "angles");
  check_terms(s.dihedrals, s.n_dihedrals, 5, f.n_dihedral_types, "dihedrals");
  for (int t = 0; t < f.n_dihedral_types; ++t) {
    if (f.dihedral_d[t] != 1 && f.dihedral_d[t] != -1) {
      throw InvalidArgument("Dihedral(\"harmonic\") dihedral_coeff.d must be +1 or -1.");
    }
    if (f.dihedral_n[t] < 0) {
      throw InvalidArgument("Dihedral(\"harmonic\") dihedral_coeff.n must be non-negative.");
    }
  }
  for (int t = 0; t < f.n_angle_types; ++t) {
    if (f.angle_theta0_deg[t] < 0.0 || f.angle_theta0_deg[t] > 180.0) {
      throw InvalidArgument(
          "Angle(\"harmonic\") angle_coeff.theta0 must be between 0 and 180 degrees.");
    }
  }
  if (f.exclusion_distance < 0 || f.exclusion_distance > 3) {
    throw InvalidArgument("bonded exclusion distance must be 1, 2, or 3.");
  }
  if (n.max_neighbors == 0) throw InvalidArgument("neighbor max_neighbors must be positive.");
  if (n.rebuild_check_every == 0) {
    throw InvalidArgument("neighbor rebuild_check_every must be positive.");
  }
  if (n.sort_every_rebuild == 0) throw InvalidArgument("neighbor.sort_every_rebuild must be positive.");
  if (!(d.dt > 0.0) || !std::isfinite(d.dt)) {
    throw InvalidArgument("dynamics.params.dt must be finite and positive.");
  }
  if (d.thermostat == 1) {
    if (!(d.temperature >= 0.0) || !std::isfinite(d.temperature)) {
      throw InvalidArgument("Thermostat(\"berendsen\").temperature must be finite and non-negative.");
    }
    if (!(d.tau > 0.0) || !std::isfinite(d.tau)) {
      throw InvalidArgument("Thermostat(\"berendsen\").tau must be finite and positive.");
    }
  }
}

std::vector<std::pair<uint32_t, uint32_t>> bond_graph_exclusions(
    uint32_t n_particles, const uint32_t* bonds, uint32_t n_bonds,
    uint32_t distance) {
  if (distance < 1 || distance > 3) {
    throw InvalidArgument("bond graph exclusion distance must be 1, 2, or 3.");
  }
  // adjacency (CSR over 1-based tags)
  std::vector<uint32_t> deg(n_particles + 2, 0);
  for (uint32_t k = 0; k < n_bonds; ++k) {
    const uint32_t a = bonds[3 * (size_t)k], b = bonds[3 * (size_t)k + 1];
    if (a == b) throw InvalidArgument("bonds entries must reference distinct tags");
    ++deg[a];
    ++deg[b];
  }
  std::vector<uint32_t> off(n_particles + 2, 0);
  for (uint32_t t = 1; t <= n_particles; ++t) off[t + 1] = off[t] + deg[t];
  std::vector<uint32_t> adj(off[n_particles + 1]);
  std::vector<uint32_t> fill(off.begin(), off.end());
  for (uint32_t k = 0; k < n_bonds; ++k) {
    const uint32_t a = bonds[3 * (size_t)k], b = bonds[3 * (size_t)k + 1];
    adj[fill[a]++] = b;
    adj[fill[b]++] = a;
  }
  // Depth-limited breadth-first search from every tag; a partner at graph
  // distance 1..d is excluded.  Canonical pairs (small, large) are kept once.
  std::vector<std::pair<uint32_t, uint32_t>> pairs;
  std::vector<uint32_t> mark(n_particles + 1, 0);
  std::vector<uint32_t> frontier, next;
  for (uint32_t s = 1; s <= n_particles; ++s) {
    if (off[s + 1] == off[s]) continue;
    frontier.assign(1, s);
    mark[s] = s;
    for (uint32_t depth = 1; depth <= distance && !frontier.empty(); ++depth) {
      next.clear();
      for (uint32_t u : frontier) {
        for (uint32_t e = off[u]; e < off[u + 1]; ++e) {
          const uint32_t w = adj[e];
          if (mark[w] == s) continue;
          mark[w] = s;
          next.push_back(w);
          if (s < w) pairs.emplace_back(s, w);
        }
      }
      frontier.swap(next);
    }
  }
  std::sort(pairs.begin(), pairs.end());
  pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
  return pairs;
}

}  // namespace bb
