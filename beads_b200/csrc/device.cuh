// device.cuh -- data layout shared by the host engine and the kernels.
//
// Every per-particle array is indexed by SLOT.  Replicas are packed one after
// another; replica r owns slots [atom_begin, atom_begin + n_pad), of which the
// first n_atoms are real particles and the rest are inert padding that makes
// every 128-thread block belong to exactly one replica.  Positions carry the
// 0-based type in the .w lane (bit pattern of an int), velocities carry the
// mass in .w, so one 16-byte load fetches what a pair or a kick needs.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bb {

constexpr int kBlock = 128;          // threads per block of per-slot kernels
// Neighbour-list interleave width: entry k of the rows of one group of kGroup
// consecutive rows is stored contiguously (see nbr_index).
#ifndef BEADS_NBR_GROUP
#define BEADS_NBR_GROUP 32
#endif
constexpr int kGroup = BEADS_NBR_GROUP;
static_assert(kGroup == 8 || kGroup == 16 || kGroup == 32, "interleave of 8, 16 or 32 rows");
constexpr int kMaxTypes = 16;        // LJ type table held in shared memory
constexpr uint32_t kKeBuckets = 128; // fixed-point kinetic-energy buckets per replica
constexpr uint32_t kScanChunk = 4096;  // cells per block of the cell-count scan
// Coordinates of the far particle at pos[n_slots] (pads neighbour batches);
// its squared distance to any particle is ~3e36, above kFarR2.
constexpr float kFarCoord = 1.0e18f;
constexpr float kFarR2 = 1.0e36f;
// Fixed-point totals: a per-slot value v is split into floor(v) and the
// fraction in units of 2^-32, each summed in its own 64-bit integer word.
// Integer sums do not depend on the order of the additions, so totals are
// bit-identical whatever the grid, batch or block shape; the whole words
// hold any total below 2^63, the fraction words any number of slots < 2^31.
constexpr double kFixFrac = 4294967296.0;  // 2^32
constexpr double kFixLimit = 4.0e18;       // |per-slot value| at or above -> status

// status bits (ReplicaState::status)
constexpr unsigned kStatusNeighborOverflow = 1u;
constexpr unsigned kStatusNonFinite = 2u;
constexpr unsigned kStatusFixedOverflow = 4u;
constexpr unsigned kStatusCellClamp = 8u;

// accumulator lanes (ReplicaState::acc)
enum AccLane : int {
  kAccPair = 0,
  kAccBond = 1,
  kAccAngle = 2,
  kAccDihedral = 3,
  kAccVirial = 4,
  kAccKinetic = 5,
  kAccLanes = 8
};

// Immutable per-replica parameters (uploaded once).
struct ReplicaParams {
  float lo[3];
  float len[3];
  float half[3];
  float inv_len[3];
  uint32_t atom_begin;       // first slot
  uint32_t n_atoms;          // real particles
  uint32_t n_pad;            // slots incl. padding (multiple of kBlock)
  uint32_t block_begin;      // first block of this replica
  uint32_t tag_base;         // global tag index of tag 1
  uint32_t cell_begin;       // first cell (global cell numbering)
  uint32_t start_base;       // first entry in cell_start (n_cells + 1 each)
  uint32_t nc[3];            // cells per axis
  uint32_t n_cells;
  float inv_cell[3];
  float search_cut_sq;       // (rc + skin)^2 in float, neighbour inclusion
  float force_cut_sq;        // rc^2 in float, pair cutoff
  float disp_thr_sq;         // (skin / 2)^2 in float
  float skin;
  uint32_t max_neighbors;    // overflow threshold of this replica
  uint32_t check_every;
  uint32_t sort_every;
  uint32_t excl_degree;      // max exclusion partners (0 = none)
  float dt;
  int32_t thermostat;        // 0 none, 1 Berendsen
  double kt_target;          // kB * T0
  double tau;
  double dof;                // 3N - 3 (>= 0)
  double kb;
  double press_scale;
  double volume;
  uint32_t lj_offset;        // first entry of this replica's LJ table
  int32_t n_types;
  uint32_t bond_type_base, angle_type_base, dihedral_type_base;
  uint32_t staged;           // pair forces from a shared-memory stage (kernels.cu)
  uint32_t sparse;           // lists built one thread per particle (k_build_sparse)
};

// Mutable per-replica device state.
struct ReplicaState {
  unsigned long long step;          // completed physical steps
  unsigned long long builds;        // neighbour builds
  unsigned long long dangerous;     // dangerous rebuilds
  unsigned int need_rebuild;        // decision for the current step
  unsigned int reorder_now;         // physical reorder during this rebuild
  unsigned int exceeded;            // displacement flag (written by threads)
  unsigned int checks_since_build;  // scheduled checks since the last build
  unsigned int done_pre;            // last-block counters
  unsigned int done_post;
  unsigned int status;              // kStatus* bits
  unsigned int pad0;
  double lambda;                    // pending Berendsen velocity scale
  double last_kinetic;              // kinetic energy of the last post (before scaling)
  long long acc[kAccLanes];         // fixed-point totals of the current eval:
  long long acc_frac[kAccLanes];    //   whole words and 2^-32 fraction words
};

// Observables of the last evaluation of one replica (device copy).
struct ReplicaObs {
  unsigned long long step;
  double pair_pe, bond_pe, angle_pe, dihedral_pe;
  double virial;
  double ke_pre;      // kinetic energy before the Berendsen scaling
  double lambda;      // scale applied to that kinetic energy (KE = l^2 KE_pre)
  unsigned long long builds, dangerous;
  unsigned int status;
  unsigned int pad;
};

// LJ coefficients of one type pair, packed as in the reference's
// LjPairModel::DeviceCoeff (native/src/forcefield/pair/pair_lj.cu:171-192).
struct LjCoeff {
  float sigma2;
  float eps4;
  float eps24;
  float shift;
};

// Harmonic term coefficients.
struct BondCoeff { float k, r0; };
struct AngleCoeff { float k, theta0; };
struct DihedralCoeff { float k; int d; int n; int pad; };

// Bonded-term membership of one particle: kind (2 bits), role (2 bits) and
// term index (28 bits).  Stored per global tag.
constexpr uint32_t kTermBond = 1u, kTermAngle = 2u, kTermDihedral = 3u;
__host__ __device__ inline uint32_t term_pack(uint32_t kind, uint32_t role,
                                              uint32_t index) {
  return (kind << 30) | (role << 28) | index;
}

__host__ __device__ inline uint64_t nbr_index(uint32_t slot, uint32_t k,
                                              uint32_t stride) {
  return ((uint64_t)(slot / (uint32_t)kGroup) * stride + k) * kGroup +
         (slot % (uint32_t)kGroup);
}

struct DeviceView {
  // particle arrays
  float4* pos;
  float4* vel;
  float4* force;
  int4* img;
  uint32_t* tag;
  uint32_t* mol;
  float4* ref_pos;
  int4* ref_img;
  uint32_t* cross;  // net boundary crossings since the last build (see pack_cross)
  uint32_t* work_start;  // [n_replicas + 1] first work item (cell) of each rebuilding
                         // replica, then the total
  // Cell-count scan in chunks of kScanChunk cells: chunk b belongs to
  // replica scan_chunk_replica[b]; replica r's chunks start at
  // scan_chunk_first[r]; scan_chunk_sum[b] holds the chunk's count total, then
  // its exclusive prefix inside the replica.
  const uint32_t* scan_chunk_replica;
  const uint32_t* scan_chunk_first;
  uint32_t* scan_chunk_sum;
  uint32_t n_scan_chunks;
  // reorder scratch
  float4* pos2;
  float4* vel2;
  int4* img2;
  uint32_t* tag2;
  uint32_t* mol2;
  uint32_t* cell2;
  // cells
  uint32_t* cell_of_slot;
  uint32_t* cell_count;
  uint32_t* cell_cursor;
  uint32_t* cell_start;
  uint32_t* cell_atoms;
  // neighbour list
  uint32_t* nbr_count;
  uint32_t* nbr;
  uint32_t nbr_stride;       // allocated capacity per slot
  // identity
  uint32_t* slot_of_tag;     // by global tag index
  // exclusions
  uint32_t* excl_slot;       // [slot * excl_cap + e]
  uint32_t excl_cap;
  const uint32_t* excl_off;  // by global tag index (+1)
  const uint32_t* excl_tag;  // partner global tag indices
  // bonded
  const uint32_t* term_off;  // by global tag index (+1)
  const uint32_t* term;      // packed memberships
  const uint4* bonds;        // (tag_i, tag_j, type, 0) global tags, global type
  const uint4* angles;       // (tag_i, tag_j, tag_k, type)
  const uint4* dihedrals;    // (tag_i, tag_j, tag_k, tag_l)
  const uint32_t* dihedral_type;
  uint32_t n_bond_terms, n_angle_terms, n_dihedral_terms;
  // term_mem: membership entry (index into term / term_off ranges) of every
  // (term, member): bonds [2 nb], then angles [3 na], then dihedrals [4 nd].
  const uint32_t* term_mem;
  float4* bonded_contrib;    // per membership entry: force on the member, energy (first member)
  float* bonded_vir;         // per membership entry: the term's virial (first member)
  const BondCoeff* bond_coeff;
  const AngleCoeff* angle_coeff;
  const DihedralCoeff* dihedral_coeff;
  // replicas
  const ReplicaParams* rp;
  ReplicaState* rs;
  ReplicaObs* obs;
  const uint32_t* block_replica;
  // Rebuild chain over the rebuilding replicas' slot blocks (batches):
  // chain_block_start[q] = blocks of the rebuilding replicas before q
  // ([n_replicas + 1], laid out by k_chain_blocks).
  uint32_t* chain_block_start;
  uint32_t chain_block_list;
  const uint32_t* cell_replica;  // replica of each global cell
  unsigned long long* chain_launches;  // launches of the rebuild chain so far
  long long* ke_part;            // [replica][kKeBuckets][whole, frac] kinetic-energy buckets
  const LjCoeff* lj;
  uint32_t n_replicas;
  // Staged context: list rows (and counts) by cell-order index of the last
  // build, entries of staged groups are stage indices; stage_cap is the
  // stage capacity in entries of a group (shared memory of k_lj_staged).
  int list_by_q;
  uint32_t stage_cap;
  uint32_t n_slots;
  uint32_t n_blocks;
  uint32_t total_cells;
  int has_bonded;
};

}  // namespace bb
