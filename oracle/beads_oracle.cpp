// beads_oracle.cpp -- CPU restatement of the BEADS per-step hot path.
//
// TEST INFRASTRUCTURE ONLY.  This library is the checker the CUDA engine is
// compared against (tests, __graft_entry__.smoke) and the CPU arm of the
// benchmark.  The product (beads_b200) never links, loads or calls it.
//
// What it restates (paths inside the reference project):
//   plan            native/src/simulation/neighbor/neighbor_plan.cpp:29-236
//   cell id         native/src/simulation/neighbor/cell_list_build.cu:110-166
//   neighbour rule  native/src/simulation/neighbor/full/full_neighbor_path_common.cuh:49-94
//                   (stencils: regular_cell_neighbor_builder.cu:40-113,
//                    small_dimension_neighbor_builder.cu:56-142,
//                    direct_neighbor_builder.cu:12-53)
//   exclusions      native/src/system/topology/exclusions.cu:514-598
//   LJ              native/src/forcefield/pair/pair_lj.cu:21-192
//   bond            native/src/forcefield/bond/bond_harmonic.cu:24-99
//   angle           native/src/forcefield/angle/angle_harmonic.cu:23-178, 238-253
//   dihedral        native/src/forcefield/dihedral/dihedral_harmonic.cu:22-227, 293-320
//   integrator      native/src/dynamics/integrator/velocity_verlet.cu:59-111
//   Berendsen       native/src/dynamics/thermostat/berendsen_thermostat.cu:104-163
//   rebuild policy  native/src/simulation/neighbor/neighbor_system.cpp:79-216,
//                   native/src/simulation/neighbor/rebuild_tracker.cu:50-94
//   thermo          native/src/system/units/unit_system.hpp:27-49,
//                   native/src/simulation/output/thermo/thermo_output.cu:46-49
//
// Precision contract:
//   * discrete decisions that the reference takes in float (cell index,
//     neighbour inclusion r^2 <= (rc+skin)^2) are evaluated in float with the
//     same operation order the CUDA engine documents: d = xi - xj, one shift by
//     L, r^2 = fma(dz,dz, fma(dx,dx, dy*dy)) (the contraction nvcc gives the
//     reference's dx * dx + dy * dy + dz * dz, pinned by its own neighbour lists);
//   * the pair-cutoff decision r^2 < rc^2 is taken in float on the exactly
//     rounded minimum-image difference (the engine's rule), so float and
//     double evaluations include the same pairs;
//   * every force, energy and virial value is computed in double from the
//     exact (double) minimum-image difference of the float coordinates.
// Built with -ffp-contract=off so that only the explicit fmaf calls fuse.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;

struct Box {
  double lo[3], len[3], half[3];
  float flo[3], flen[3], fhalf[3], finv[3];
};

Box make_box(const float lo[3], const float hi[3]) {
  Box b;
  for (int a = 0; a < 3; ++a) {
    b.flo[a] = lo[a];
    b.flen[a] = hi[a] - lo[a];
    b.fhalf[a] = 0.5f * b.flen[a];
    b.finv[a] = 1.0f / b.flen[a];
    b.lo[a] = b.flo[a];
    b.len[a] = b.flen[a];
    b.half[a] = b.fhalf[a];
  }
  return b;
}

// Reference rule in float (one subtraction, one shift).
inline float ref_delta_f(float xi, float xj, float len, float half) {
  float d = xi - xj;
  if (d > half) d -= len;
  else if (d < -half) d += len;
  return d;
}

// Exact minimum-image difference of two float coordinates, in double.  The
// subtraction and the shift are exact in double for float inputs.
inline double exact_delta(float xi, float xj, double len, double half) {
  double d = static_cast<double>(xi) - static_cast<double>(xj);
  if (d > half) d -= len;
  else if (d < -half) d += len;
  return d;
}

inline float norm2_f(float dx, float dy, float dz) {
  return std::fmaf(dz, dz, std::fmaf(dx, dx, dy * dy));
}

uint32_t axis_cell(float x, float lo, float inv, uint32_t n) {
  const float scaled = (x - lo) * inv;
  if (scaled <= 0.0f) return 0u;
  if (scaled >= static_cast<float>(n)) return n - 1u;
  const uint32_t i = static_cast<uint32_t>(scaled);
  return i >= n ? n - 1u : i;
}

int stencil(uint32_t c, uint32_t n, uint32_t out[3]) {
  if (n <= 1u) { out[0] = 0; return 1; }
  if (n == 2u) { out[0] = 0; out[1] = 1; return 2; }
  out[0] = c == 0 ? n - 1 : c - 1;
  out[1] = c;
  out[2] = c + 1 == n ? 0 : c + 1;
  return 3;
}

struct Plan {
  uint32_t nc[3];
  float inv_cell[3];
  float search;
  float search_sq;
  int path;
};

int make_plan(const float lo[3], const float hi[3], double cutoff, double skin, Plan* p) {
  const float rc = static_cast<float>(cutoff);
  const float sk = static_cast<float>(skin);
  p->search = rc + sk;
  p->search_sq = p->search * p->search;
  float len[3];
  float shortest = 0;
  for (int a = 0; a < 3; ++a) {
    len[a] = hi[a] - lo[a];
    shortest = a == 0 ? len[a] : std::min(shortest, len[a]);
  }
  if (p->search > 0.5f * shortest) return -1;
  for (int a = 0; a < 3; ++a) {
    const double raw = std::floor(static_cast<double>(len[a]) / static_cast<double>(p->search));
    p->nc[a] = raw < 1.0 ? 1u : static_cast<uint32_t>(raw);
    const float cell = len[a] / static_cast<float>(p->nc[a]);
    p->inv_cell[a] = 1.0f / cell;
  }
  const bool small = p->nc[0] < 3 && p->nc[1] < 3 && p->nc[2] < 3;
  const bool large = p->nc[0] >= 3 && p->nc[1] >= 3 && p->nc[2] >= 3;
  p->path = small ? 0 : (large ? 1 : 2);
  return 0;
}

// Cell list of float positions (reference cell rule).
struct Cells {
  std::vector<uint32_t> cell_of, start, atoms;
};

void bin(uint32_t n, const float* pos, const Box& b, const Plan& p, Cells* c) {
  const uint32_t ncell = p.nc[0] * p.nc[1] * p.nc[2];
  c->cell_of.resize(n);
  c->start.assign(ncell + 1, 0);
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t ix = axis_cell(pos[3 * i], b.flo[0], p.inv_cell[0], p.nc[0]);
    const uint32_t iy = axis_cell(pos[3 * i + 1], b.flo[1], p.inv_cell[1], p.nc[1]);
    const uint32_t iz = axis_cell(pos[3 * i + 2], b.flo[2], p.inv_cell[2], p.nc[2]);
    c->cell_of[i] = ix + p.nc[0] * (iy + p.nc[1] * iz);
    c->start[c->cell_of[i] + 1]++;
  }
  for (uint32_t k = 0; k < ncell; ++k) c->start[k + 1] += c->start[k];
  c->atoms.resize(n);
  std::vector<uint32_t> cur(c->start.begin(), c->start.end() - 1);
  for (uint32_t i = 0; i < n; ++i) c->atoms[cur[c->cell_of[i]]++] = i;
}

// Full neighbour lists, reference inclusion rule on float positions.  Sorted
// by partner row.  Exclusions: CSR over rows (partners by row index).
void neighbors_f(uint32_t n, const float* pos, const Box& b, const Plan& p,
                 const uint32_t* ex_off, const uint32_t* ex_idx,
                 std::vector<std::vector<uint32_t>>* out) {
  Cells c;
  bin(n, pos, b, p, &c);
  out->assign(n, {});
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t ii = 0; ii < static_cast<int64_t>(n); ++ii) {
    const uint32_t i = static_cast<uint32_t>(ii);
    const uint32_t cell = c.cell_of[i];
    const uint32_t cx = cell % p.nc[0], cy = (cell / p.nc[0]) % p.nc[1], cz = cell / (p.nc[0] * p.nc[1]);
    uint32_t sx[3], sy[3], sz[3];
    const int nx = stencil(cx, p.nc[0], sx), ny = stencil(cy, p.nc[1], sy), nz = stencil(cz, p.nc[2], sz);
    std::vector<uint32_t>& row = (*out)[i];
    for (int a = 0; a < nz; ++a)
      for (int bb = 0; bb < ny; ++bb)
        for (int cc = 0; cc < nx; ++cc) {
          const uint32_t lc = sx[cc] + p.nc[0] * (sy[bb] + p.nc[1] * sz[a]);
          for (uint32_t q = c.start[lc]; q < c.start[lc + 1]; ++q) {
            const uint32_t j = c.atoms[q];
            if (j == i) continue;
            bool excluded = false;
            if (ex_off) {
              for (uint32_t e = ex_off[i]; e < ex_off[i + 1]; ++e) excluded |= ex_idx[e] == j;
            }
            if (excluded) continue;
            const float dx = ref_delta_f(pos[3 * i], pos[3 * j], b.flen[0], b.fhalf[0]);
            const float dy = ref_delta_f(pos[3 * i + 1], pos[3 * j + 1], b.flen[1], b.fhalf[1]);
            const float dz = ref_delta_f(pos[3 * i + 2], pos[3 * j + 2], b.flen[2], b.fhalf[2]);
            if (norm2_f(dx, dy, dz) > p.search_sq) continue;
            row.push_back(j);
          }
        }
    std::sort(row.begin(), row.end());
  }
}

// ---- force field -----------------------------------------------------------
struct FF {
  int ntypes;
  const double* eps;
  const double* sig;
  double rc;
  int shift;
  uint32_t nb;
  const uint32_t* bonds;       // [nb][3] rows are 0-based particle rows
  const double* bond_k;
  const double* bond_r0;
  uint32_t na;
  const uint32_t* angles;      // [na][4]
  const double* angle_k;
  const double* angle_theta0_deg;
  uint32_t nd;
  const uint32_t* dihedrals;   // [nd][5]
  const double* dihedral_k;
  const int32_t* dihedral_d;
  const int32_t* dihedral_n;
  // Steepest-descent form only: LJ evaluated on r^2 clamped to at least
  // clamp_sig2 * sigma^2 (0 = the plain pair force).
  double clamp_sig2 = 0.0;
};

struct Out {
  double pair = 0, bond = 0, angle = 0, dihedral = 0, virial = 0;
};

struct D3 {
  double x, y, z;
};
inline D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 mul(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

D3 arm(const float* pos, const Box& b, uint32_t i, uint32_t j) {
  return {exact_delta(pos[3 * i], pos[3 * j], b.len[0], b.half[0]),
          exact_delta(pos[3 * i + 1], pos[3 * j + 1], b.len[1], b.half[1]),
          exact_delta(pos[3 * i + 2], pos[3 * j + 2], b.len[2], b.half[2])};
}

// Pair forces over full neighbour lists (each pair seen from both ends).
void pair_forces(uint32_t n, const float* pos, const int32_t* types, const Box& b, const FF& ff,
                 const std::vector<std::vector<uint32_t>>& nbr, double* f, Out* out) {
  const float rcf = static_cast<float>(ff.rc);
  const float rc2f = rcf * rcf;
  const double rc2 = static_cast<double>(rcf) * static_cast<double>(rcf);
  double pe = 0.0, vir = 0.0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : pe, vir)
  for (int64_t ii = 0; ii < static_cast<int64_t>(n); ++ii) {
    const uint32_t i = static_cast<uint32_t>(ii);
    double fx = 0, fy = 0, fz = 0, e = 0, w = 0;
    const int ti = types[i] - 1;
    for (uint32_t j : nbr[i]) {
      const D3 d = arm(pos, b, i, j);
      const float r2f = norm2_f(static_cast<float>(d.x), static_cast<float>(d.y), static_cast<float>(d.z));
      if (!(r2f < rc2f)) continue;
      const int tj = types[j] - 1;
      const double eps = ff.eps[ti * ff.ntypes + tj];
      const double sig = ff.sig[ti * ff.ntypes + tj];
      double r2 = dot(d, d);
      if (ff.clamp_sig2 > 0.0) r2 = std::max(r2, ff.clamp_sig2 * sig * sig);
      const double sr2 = sig * sig / r2;
      const double sr6 = sr2 * sr2 * sr2;
      const double sr12 = sr6 * sr6;
      const double fs = 24.0 * eps / r2 * (2.0 * sr12 - sr6);
      fx += fs * d.x;
      fy += fs * d.y;
      fz += fs * d.z;
      double shift = 0.0;
      if (ff.shift) {
        const double s2 = sig * sig / rc2;
        const double s6 = s2 * s2 * s2;
        shift = 4.0 * eps * (s6 * s6 - s6);
      }
      e += 4.0 * eps * (sr12 - sr6) - shift;
      w += fs * r2;
    }
    f[3 * i] += fx;
    f[3 * i + 1] += fy;
    f[3 * i + 2] += fz;
    pe += 0.5 * e;
    vir += 0.5 * w;
  }
  out->pair += pe;
  out->virial += vir;
}

void bonded_forces(const float* pos, const Box& b, const FF& ff, double* f, Out* out) {
  for (uint32_t k = 0; k < ff.nb; ++k) {
    const uint32_t i = ff.bonds[3 * k], j = ff.bonds[3 * k + 1];
    const int t = ff.bonds[3 * k + 2] - 1;
    const D3 d = arm(pos, b, i, j);
    const double r = std::sqrt(dot(d, d));
    const double s = r - ff.bond_r0[t];
    out->bond += 0.5 * ff.bond_k[t] * s * s;
    if (r == 0.0) continue;
    const double sc = -ff.bond_k[t] * s / r;
    const D3 fi = mul(sc, d);
    f[3 * i] += fi.x; f[3 * i + 1] += fi.y; f[3 * i + 2] += fi.z;
    f[3 * j] -= fi.x; f[3 * j + 1] -= fi.y; f[3 * j + 2] -= fi.z;
    out->virial += dot(d, fi);
  }
  for (uint32_t k = 0; k < ff.na; ++k) {
    const uint32_t i = ff.angles[4 * k], j = ff.angles[4 * k + 1], m = ff.angles[4 * k + 2];
    const int t = ff.angles[4 * k + 3] - 1;
    const double kk = ff.angle_k[t];
    const double th0 = ff.angle_theta0_deg[t] * kPi / 180.0;
    const D3 a1 = arm(pos, b, i, j), a2 = arm(pos, b, m, j);
    const double q1 = dot(a1, a1), q2 = dot(a2, a2);
    if (q1 == 0.0 || q2 == 0.0) {
      out->angle += 0.5 * kk * th0 * th0;
      continue;
    }
    const double r1 = std::sqrt(q1), r2 = std::sqrt(q2);
    double cs = std::min(1.0, std::max(-1.0, dot(a1, a2) / (r1 * r2)));
    const double th = std::acos(cs);
    const double dth = th - th0;
    out->angle += 0.5 * kk * dth * dth;
    const double s2 = 1.0 - cs * cs;
    const double sn = s2 <= 1.0e-6 ? 1.0e-3 : std::sqrt(s2);
    const double a = -kk * dth / sn;
    const double c11 = a * cs / q1, c12 = -a / (r1 * r2), c22 = a * cs / q2;
    const D3 fi = add(mul(c11, a1), mul(c12, a2));
    const D3 fk = add(mul(c22, a2), mul(c12, a1));
    f[3 * i] += fi.x; f[3 * i + 1] += fi.y; f[3 * i + 2] += fi.z;
    f[3 * m] += fk.x; f[3 * m + 1] += fk.y; f[3 * m + 2] += fk.z;
    f[3 * j] -= fi.x + fk.x; f[3 * j + 1] -= fi.y + fk.y; f[3 * j + 2] -= fi.z + fk.z;
    out->virial += dot(a1, fi) + dot(a2, fk);
  }
  for (uint32_t k = 0; k < ff.nd; ++k) {
    const uint32_t i = ff.dihedrals[5 * k], j = ff.dihedrals[5 * k + 1];
    const uint32_t m = ff.dihedrals[5 * k + 2], l = ff.dihedrals[5 * k + 3];
    const int t = ff.dihedrals[5 * k + 4] - 1;
    const double kk = ff.dihedral_k[t];
    const double dd = ff.dihedral_d[t];
    const int nn = ff.dihedral_n[t];
    const D3 b0 = arm(pos, b, i, j), b1 = arm(pos, b, m, j), b2 = arm(pos, b, m, l);
    const D3 u = cross(b0, b1), w = cross(b1, b2);
    const double q1 = dot(b1, b1), qu = dot(u, u), qw = dot(w, w);
    if (q1 == 0.0 || qu == 0.0 || qw == 0.0) {
      out->dihedral += nn == 0 ? kk * (1.0 + dd) : kk;
      continue;
    }
    double cs = std::min(1.0, std::max(-1.0, dot(u, w) / std::sqrt(qu * qw)));
    double phi = std::acos(cs);
    if (dot(b0, w) < 0.0) phi = -phi;
    out->dihedral += kk * (1.0 + dd * std::cos(nn * phi));
    const double de = -kk * dd * nn * std::sin(nn * phi);
    const double l1 = std::sqrt(q1);
    const D3 fi = mul(-de * l1 / qu, u);
    const D3 fl = mul(de * l1 / qw, w);
    const D3 s = sub(mul(dot(b0, b1) / q1, fi), mul(dot(b2, b1) / q1, fl));
    const D3 fj = sub(s, fi);
    const D3 fk = mul(-1.0, add(s, fl));
    f[3 * i] += fi.x; f[3 * i + 1] += fi.y; f[3 * i + 2] += fi.z;
    f[3 * j] += fj.x; f[3 * j + 1] += fj.y; f[3 * j + 2] += fj.z;
    f[3 * m] += fk.x; f[3 * m + 1] += fk.y; f[3 * m + 2] += fk.z;
    f[3 * l] += fl.x; f[3 * l + 1] += fl.y; f[3 * l + 2] += fl.z;
    out->virial += dot(b0, fi) + dot(b1, fk) + dot(sub(b1, b2), fl);
  }
}

void exclusion_csr(uint32_t n, const FF& ff, int distance, std::vector<uint32_t>* off,
                   std::vector<uint32_t>* idx);

}  // namespace

extern "C" {

// Plan of one box: cells per axis, inverse cell size (float), search cutoff
// squared (float), path 0 direct / 1 regular_cell / 2 small_dimension.
// Returns -1 if rc + skin exceeds half the shortest box length.
int orc_plan(const float lo[3], const float hi[3], double cutoff, double skin, uint32_t nc[3],
             float inv_cell[3], float* search_sq, int* path) {
  Plan p;
  if (make_plan(lo, hi, cutoff, skin, &p) != 0) return -1;
  for (int a = 0; a < 3; ++a) {
    nc[a] = p.nc[a];
    inv_cell[a] = p.inv_cell[a];
  }
  *search_sq = p.search_sq;
  *path = p.path;
  return 0;
}

void orc_cell_ids(uint32_t n, const float* pos, const float lo[3], const float hi[3],
                  double cutoff, double skin, uint32_t* cell_out) {
  Plan p;
  make_plan(lo, hi, cutoff, skin, &p);
  const Box b = make_box(lo, hi);
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t ix = axis_cell(pos[3 * i], b.flo[0], p.inv_cell[0], p.nc[0]);
    const uint32_t iy = axis_cell(pos[3 * i + 1], b.flo[1], p.inv_cell[1], p.nc[1]);
    const uint32_t iz = axis_cell(pos[3 * i + 2], b.flo[2], p.inv_cell[2], p.nc[2]);
    cell_out[i] = ix + p.nc[0] * (iy + p.nc[1] * iz);
  }
}

// Bond-graph exclusion pairs (0-based rows, i < j, sorted).  Returns the pair
// count; writes up to max_pairs pairs.
int64_t orc_exclusions(uint32_t n, const uint32_t* bonds, uint32_t nb, uint32_t distance,
                       uint32_t* pairs, uint64_t max_pairs) {
  std::vector<std::vector<uint32_t>> adj(n);
  for (uint32_t k = 0; k < nb; ++k) {
    adj[bonds[3 * k]].push_back(bonds[3 * k + 1]);
    adj[bonds[3 * k + 1]].push_back(bonds[3 * k]);
  }
  std::vector<std::pair<uint32_t, uint32_t>> out;
  std::vector<int> dist(n, -1);
  for (uint32_t s = 0; s < n; ++s) {
    std::vector<uint32_t> seen{s};
    std::vector<uint32_t> queue{s};
    dist[s] = 0;
    for (size_t h = 0; h < queue.size(); ++h) {
      const uint32_t u = queue[h];
      if (dist[u] == static_cast<int>(distance)) continue;
      for (uint32_t w : adj[u]) {
        if (dist[w] >= 0) continue;
        dist[w] = dist[u] + 1;
        seen.push_back(w);
        queue.push_back(w);
        if (s < w) out.emplace_back(s, w);
      }
    }
    for (uint32_t u : seen) dist[u] = -1;
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  for (uint64_t k = 0; k < out.size() && k < max_pairs; ++k) {
    pairs[2 * k] = out[k].first;
    pairs[2 * k + 1] = out[k].second;
  }
  return static_cast<int64_t>(out.size());
}

// Neighbour lists of float positions.  counts[i] = full count; partners are
// sorted rows, truncated at cap per row.  ex_off/ex_idx: exclusion CSR over
// rows (may be NULL).
int orc_neighbors(uint32_t n, const float* pos, const float lo[3], const float hi[3],
                  double cutoff, double skin, const uint32_t* ex_off, const uint32_t* ex_idx,
                  uint32_t cap, uint32_t* counts, uint32_t* partners) {
  Plan p;
  if (make_plan(lo, hi, cutoff, skin, &p) != 0) return -1;
  const Box b = make_box(lo, hi);
  std::vector<std::vector<uint32_t>> nbr;
  neighbors_f(n, pos, b, p, ex_off, ex_idx, &nbr);
  for (uint32_t i = 0; i < n; ++i) {
    counts[i] = static_cast<uint32_t>(nbr[i].size());
    for (uint32_t k = 0; k < nbr[i].size() && k < cap; ++k) partners[(uint64_t)i * cap + k] = nbr[i][k];
  }
  return 0;
}

// Forces / energies / virial in double at float positions.  Particle rows are
// 0-based; bonded records use rows (tag - 1 for tag-ordered input).
// energies_out: [pair, bond, angle, dihedral]; virial_out: scalar.
int orc_forces(uint32_t n, const float* pos, const int32_t* types, const float lo[3],
               const float hi[3], int ntypes, const double* eps, const double* sig, double rc,
               int shift, double skin, int excl_distance, uint32_t nb, const uint32_t* bonds,
               const double* bond_k, const double* bond_r0, uint32_t na, const uint32_t* angles,
               const double* angle_k, const double* angle_theta0_deg, uint32_t nd,
               const uint32_t* dihedrals, const double* dihedral_k, const int32_t* dihedral_d,
               const int32_t* dihedral_n, double* force_out, double* energies_out,
               double* virial_out) {
  Plan p;
  if (make_plan(lo, hi, rc, skin, &p) != 0) return -1;
  const Box b = make_box(lo, hi);
  FF ff{ntypes, eps, sig, rc, shift, nb, bonds, bond_k, bond_r0, na, angles, angle_k,
        angle_theta0_deg, nd, dihedrals, dihedral_k, dihedral_d, dihedral_n};
  std::vector<uint32_t> ex_off, ex_idx;
  if (excl_distance > 0 && nb > 0) exclusion_csr(n, ff, excl_distance, &ex_off, &ex_idx);
  std::vector<std::vector<uint32_t>> nbr;
  neighbors_f(n, pos, b, p, ex_off.empty() ? nullptr : ex_off.data(),
              ex_idx.empty() ? nullptr : ex_idx.data(), &nbr);
  std::memset(force_out, 0, sizeof(double) * 3 * n);
  Out out;
  pair_forces(n, pos, types, b, ff, nbr, force_out, &out);
  bonded_forces(pos, b, ff, force_out, &out);
  energies_out[0] = out.pair;
  energies_out[1] = out.bond;
  energies_out[2] = out.angle;
  energies_out[3] = out.dihedral;
  *virial_out = out.virial;
  return 0;
}

// Velocity-Verlet + Berendsen state in double, advanced step by step with the
// reference's step order and rebuild policy (simulation_run.cpp:212-235,
// neighbor_system.cpp:79-105).  The neighbour list is built from the state
// rounded to float so that pair sets follow the engine's float rules; forces,
// energies and the integration are double.
struct OracleSim {
  uint32_t n = 0;
  std::vector<double> pos, vel, mass, f, ref;
  std::vector<int32_t> img, ref_img, types;
  std::vector<float> fpos;
  std::vector<uint32_t> bonds_v, angles_v, dihedrals_v;
  std::vector<double> eps_v, sig_v, bk, br0, ak, at0, dk;
  std::vector<int32_t> dd, dn;
  Plan plan{};
  Box box{};
  FF ff{};
  std::vector<uint32_t> ex_off, ex_idx;
  std::vector<std::vector<uint32_t>> nbr;
  double dt = 0, skin = 0, kt = 0, tau = 1, dof = 0, thr = 0;
  int thermostat = 0;
  uint64_t check_every = 1, builds = 0, step = 0;
  Out last;

  void to_float() {
    for (uint64_t k = 0; k < 3ull * n; ++k) fpos[k] = static_cast<float>(pos[k]);
  }
  void rebuild() {
    to_float();
    neighbors_f(n, fpos.data(), box, plan, ex_off.empty() ? nullptr : ex_off.data(),
                ex_idx.empty() ? nullptr : ex_idx.data(), &nbr);
    ref = pos;
    ref_img = img;
    ++builds;
  }
  void forces() {
    to_float();
    std::fill(f.begin(), f.end(), 0.0);
    last = Out();
    pair_forces(n, fpos.data(), types.data(), box, ff, nbr, f.data(), &last);
    bonded_forces(fpos.data(), box, ff, f.data(), &last);
  }
  double kinetic() const {
    double ke = 0;
#pragma omp parallel for reduction(+ : ke)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
      ke += 0.5 * mass[i] * (vel[3 * i] * vel[3 * i] + vel[3 * i + 1] * vel[3 * i + 1] +
                             vel[3 * i + 2] * vel[3 * i + 2]);
    }
    return ke;
  }
  void advance() {
    ++step;
#pragma omp parallel for
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
      const double h = 0.5 * dt / mass[i];
      for (int a = 0; a < 3; ++a) {
        double& v = vel[3 * i + a];
        double& x = pos[3 * i + a];
        v += h * f[3 * i + a];
        x += dt * v;
        const double c = std::floor((x - box.lo[a]) / box.len[a]);
        x -= c * box.len[a];
        img[3 * i + a] += static_cast<int32_t>(c);
      }
    }
    bool need = skin == 0.0;
    if (!need && step % check_every == 0) {
      int exceeded = 0;
#pragma omp parallel for reduction(| : exceeded)
      for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
        double d2 = 0;
        for (int a = 0; a < 3; ++a) {
          const double d = pos[3 * i + a] - ref[3 * i + a] +
                           static_cast<double>(img[3 * i + a] - ref_img[3 * i + a]) * box.len[a];
          d2 += d * d;
        }
        exceeded |= d2 > thr ? 1 : 0;
      }
      need = exceeded != 0;
    }
    if (need) rebuild();
    forces();
#pragma omp parallel for
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
      const double h = 0.5 * dt / mass[i];
      for (int a = 0; a < 3; ++a) vel[3 * i + a] += h * f[3 * i + a];
    }
    if (thermostat == 1) {
      const double ke = kinetic();
      double lam = 1.0;
      if (ke > 0.0 && dof > 0.0) {
        const double arg = 1.0 + dt / tau * (kt / (2.0 * ke / dof) - 1.0);
        lam = std::sqrt(std::max(0.0, arg));
      }
      for (uint64_t k = 0; k < 3ull * n; ++k) vel[k] *= lam;
    }
  }
};

}  // extern "C"

template <typename T>
static std::vector<T> copy_of(const T* p, size_t count) {
  return p ? std::vector<T>(p, p + count) : std::vector<T>();
}

extern "C" {

// Creates a simulation state (initial list + forces computed).
void* orc_sim_create(uint32_t n, const double* pos, const double* vel, const double* mass,
                     const int32_t* img, const int32_t* types, const float lo[3],
                     const float hi[3], int ntypes, const double* eps, const double* sig,
                     double rc, int shift, double skin, uint64_t check_every, int excl_distance,
                     uint32_t nb, const uint32_t* bonds, const double* bond_k,
                     const double* bond_r0, uint32_t na, const uint32_t* angles,
                     const double* angle_k, const double* angle_theta0_deg, uint32_t nd,
                     const uint32_t* dihedrals, const double* dihedral_k,
                     const int32_t* dihedral_d, const int32_t* dihedral_n, double dt,
                     int thermostat, double kt_target, double tau) {
  auto* s = new OracleSim;
  if (make_plan(lo, hi, rc, skin, &s->plan) != 0) {
    delete s;
    return nullptr;
  }
  s->n = n;
  s->box = make_box(lo, hi);
  s->pos.assign(pos, pos + 3ull * n);
  s->vel.assign(vel, vel + 3ull * n);
  s->mass.assign(mass, mass + n);
  s->img = img ? std::vector<int32_t>(img, img + 3ull * n) : std::vector<int32_t>(3ull * n, 0);
  s->types.assign(types, types + n);
  s->fpos.resize(3ull * n);
  s->f.assign(3ull * n, 0.0);
  s->eps_v.assign(eps, eps + ntypes * ntypes);
  s->sig_v.assign(sig, sig + ntypes * ntypes);
  s->bonds_v = copy_of(bonds, 3ull * nb);
  s->angles_v = copy_of(angles, 4ull * na);
  s->dihedrals_v = copy_of(dihedrals, 5ull * nd);
  int nbt = 0, nat = 0, ndt = 0;
  for (uint32_t k = 0; k < nb; ++k) nbt = std::max<int>(nbt, bonds[3 * k + 2]);
  for (uint32_t k = 0; k < na; ++k) nat = std::max<int>(nat, angles[4 * k + 3]);
  for (uint32_t k = 0; k < nd; ++k) ndt = std::max<int>(ndt, dihedrals[5 * k + 4]);
  s->bk = copy_of(bond_k, nbt);
  s->br0 = copy_of(bond_r0, nbt);
  s->ak = copy_of(angle_k, nat);
  s->at0 = copy_of(angle_theta0_deg, nat);
  s->dk = copy_of(dihedral_k, ndt);
  s->dd = copy_of(dihedral_d, ndt);
  s->dn = copy_of(dihedral_n, ndt);
  s->ff = FF{ntypes, s->eps_v.data(), s->sig_v.data(), rc, shift,
             nb, s->bonds_v.data(), s->bk.data(), s->br0.data(),
             na, s->angles_v.data(), s->ak.data(), s->at0.data(),
             nd, s->dihedrals_v.data(), s->dk.data(), s->dd.data(), s->dn.data()};
  if (excl_distance > 0 && nb > 0) exclusion_csr(n, s->ff, excl_distance, &s->ex_off, &s->ex_idx);
  s->dt = dt;
  s->skin = skin;
  s->check_every = check_every;
  s->thermostat = thermostat;
  s->kt = kt_target;
  s->tau = tau;
  s->dof = std::max(0.0, 3.0 * n - 3.0);
  const double sk = static_cast<double>(static_cast<float>(skin));
  s->thr = 0.25 * sk * sk;
  s->rebuild();
  s->forces();
  return s;
}

void orc_sim_destroy(void* sim) { delete static_cast<OracleSim*>(sim); }

// Capped steepest descent of the state's positions (velocities untouched),
// the engine's relaxation of random starts restated in double: per iteration
// forces at the current positions with LJ on r^2 clamped to >= 0.49 sigma^2,
// every particle moved by dmax * F / max(|F|, fref), wrapped, and the list
// rebuilt when a displacement since the last build exceeds skin / 2.
// Afterwards the list and the plain forces are rebuilt and the step and build
// counters restart, as for a fresh run.
void orc_sim_minimize(void* sim, uint32_t iterations, double dmax, double fref) {
  auto* s = static_cast<OracleSim*>(sim);
  s->ff.clamp_sig2 = 0.49;
  s->rebuild();
  for (uint32_t it = 0; it < iterations; ++it) {
    s->forces();
    const Box& box = s->box;
#pragma omp parallel for
    for (int64_t i = 0; i < static_cast<int64_t>(s->n); ++i) {
      const double fx = s->f[3 * i], fy = s->f[3 * i + 1], fz = s->f[3 * i + 2];
      const double fn = std::sqrt(fx * fx + fy * fy + fz * fz);
      const double k = dmax / std::max(fn, fref);
      if (!std::isfinite(k) || !std::isfinite(fn)) continue;
      for (int a = 0; a < 3; ++a) {
        double& x = s->pos[3 * i + a];
        x += k * s->f[3 * i + a];
        const double c = std::floor((x - box.lo[a]) / box.len[a]);
        x -= c * box.len[a];
        s->img[3 * i + a] += static_cast<int32_t>(c);
      }
    }
    int exceeded = 0;
#pragma omp parallel for reduction(| : exceeded)
    for (int64_t i = 0; i < static_cast<int64_t>(s->n); ++i) {
      double d2 = 0;
      for (int a = 0; a < 3; ++a) {
        const double d = s->pos[3 * i + a] - s->ref[3 * i + a] +
                         static_cast<double>(s->img[3 * i + a] - s->ref_img[3 * i + a]) *
                             box.len[a];
        d2 += d * d;
      }
      exceeded |= d2 > s->thr ? 1 : 0;
    }
    if (exceeded) s->rebuild();
  }
  s->ff.clamp_sig2 = 0.0;
  s->rebuild();
  s->forces();
  s->builds = 0;
  s->step = 0;
}

// Advances `steps`; writes the observables of the last force evaluation:
// [step, pair, bond, angle, dihedral, ke, virial] (ke after Berendsen).
void orc_sim_step(void* sim, uint64_t steps, double* obs) {
  auto* s = static_cast<OracleSim*>(sim);
  for (uint64_t k = 0; k < steps; ++k) s->advance();
  if (obs) {
    obs[0] = static_cast<double>(s->step);
    obs[1] = s->last.pair;
    obs[2] = s->last.bond;
    obs[3] = s->last.angle;
    obs[4] = s->last.dihedral;
    obs[5] = s->kinetic();
    obs[6] = s->last.virial;
  }
}

void orc_sim_state(void* sim, double* pos, double* vel, int32_t* img, uint64_t* builds) {
  auto* s = static_cast<OracleSim*>(sim);
  if (pos) std::memcpy(pos, s->pos.data(), sizeof(double) * 3 * s->n);
  if (vel) std::memcpy(vel, s->vel.data(), sizeof(double) * 3 * s->n);
  if (img) std::memcpy(img, s->img.data(), sizeof(int32_t) * 3 * s->n);
  if (builds) *builds = s->builds;
}

int orc_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"

namespace {

void exclusion_csr(uint32_t n, const FF& ff, int distance, std::vector<uint32_t>* off,
                   std::vector<uint32_t>* idx) {
  std::vector<uint32_t> pairs;
  const int64_t cnt = orc_exclusions(n, ff.bonds, ff.nb, distance, nullptr, 0);
  pairs.resize(2 * static_cast<size_t>(cnt));
  orc_exclusions(n, ff.bonds, ff.nb, distance, pairs.data(), cnt);
  std::vector<std::vector<uint32_t>> rows(n);
  for (int64_t k = 0; k < cnt; ++k) {
    rows[pairs[2 * k]].push_back(pairs[2 * k + 1]);
    rows[pairs[2 * k + 1]].push_back(pairs[2 * k]);
  }
  off->assign(n + 1, 0);
  for (uint32_t i = 0; i < n; ++i) (*off)[i + 1] = (*off)[i] + static_cast<uint32_t>(rows[i].size());
  idx->clear();
  for (uint32_t i = 0; i < n; ++i) idx->insert(idx->end(), rows[i].begin(), rows[i].end());
}

}  // namespace
