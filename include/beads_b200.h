/*
 * beads_b200.h -- C ABI of the B200-native BEADS molecular-dynamics engine.
 *
 * The reference binds its engine through one pybind11 module, `beads._native`,
 * with two functions (native/src/bindings/module.cpp:15-55):
 *   build_info()             -> dict of dtype names
 *   execute_simulation(spec) -> None, results go to files
 * This header is the plain-C boundary underneath a drop-in replacement for that
 * module.  Every entry point takes plain pointers and sizes; no C++ or torch
 * type crosses it.  All functions return 0 (BEADS_OK) on success or a negative
 * status; the message of the last failure on the calling thread is available
 * through beads_last_error().  Status codes map onto the Python exception types
 * the reference raises (ValueError / RuntimeError / OverflowError).
 *
 * Terms:
 *   replica  -- one independent periodic system (box, particles, topology).
 *               A single simulation is a batch of one replica.
 *   slot     -- the device storage position of a particle; slots are permuted
 *               by the cell sort.  Every host-facing array in this header is in
 *               TAG order (index = tag - 1) unless it says otherwise.
 *   real     -- float (IEEE binary32): positions, velocities, masses and forces
 *               are float, as in the reference's default single-precision build
 *               (native/include/beads/core/types.hpp:12-20).
 */
#ifndef BEADS_B200_H
#define BEADS_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define BEADS_API __attribute__((visibility("default")))
#else
#define BEADS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define BEADS_OK 0
#define BEADS_ERR_INVALID (-1)   /* bad argument / spec  -> ValueError       */
#define BEADS_ERR_RUNTIME (-2)   /* runtime failure      -> RuntimeError     */
#define BEADS_ERR_OVERFLOW (-3)  /* size / range overflow-> OverflowError    */
#define BEADS_ERR_CUDA (-4)      /* CUDA error           -> RuntimeError     */
#define BEADS_ERR_NEIGHBOR_OVERFLOW (-5) /* list overflow -> RuntimeError    */
#define BEADS_ERR_NONFINITE (-6) /* non-finite force/energy -> RuntimeError  */
#define BEADS_ERR_INTERRUPTED (-7) /* interrupt callback asked to stop       */

/* ---- units (native/src/system/units/unit_system.cpp:9-12) --------------- */
#define BEADS_UNITS_REDUCED 0
#define BEADS_UNITS_NM_KJMOL 1

/* ---- trajectory field mask (native/src/simulation/output/trajectory/
 *      trajectory_output.cu:38-45) ---------------------------------------- */
#define BEADS_FIELD_TAG (1u << 0)
#define BEADS_FIELD_TYPE (1u << 1)
#define BEADS_FIELD_POSITION (1u << 2)
#define BEADS_FIELD_IMAGE (1u << 3)
#define BEADS_FIELD_VELOCITY (1u << 4)
#define BEADS_FIELD_FORCE (1u << 5)

/* ---- log echo modes (native/src/simulation/output/log/log_output.cpp) --- */
#define BEADS_ECHO_NONE 0
#define BEADS_ECHO_SCREEN 1
#define BEADS_ECHO_LOG 2
#define BEADS_ECHO_BOTH 3

/* One replica's particles, box and topology.  Replaces input::SystemSpec
 * (native/src/input/native_spec.hpp:51-62).  Arrays are in the caller's
 * order; `tags` gives each row's tag (a permutation of 1..n), NULL = 1..n. */
typedef struct beads_system_desc {
  uint32_t n_particles;
  int32_t units;                 /* BEADS_UNITS_*                              */
  float box_lo[3];
  float box_hi[3];
  const float* positions;        /* [n][3], inside [lo, hi)                    */
  const float* velocities;       /* [n][3] or NULL (zero)                      */
  const float* masses;           /* [n] or NULL (one)                          */
  const int32_t* types;          /* [n], dense 1-based                         */
  const uint32_t* tags;          /* [n] or NULL                                */
  const uint32_t* molecule_ids;  /* [n] or NULL (one)                          */
  const int32_t* images;         /* [n][3] or NULL (zero)                      */
  uint32_t n_bonds;
  const uint32_t* bonds;         /* [n_bonds][3]: tag_i, tag_j, type           */
  uint32_t n_angles;
  const uint32_t* angles;        /* [n_angles][4]: tag_i, tag_j, tag_k, type   */
  uint32_t n_dihedrals;
  const uint32_t* dihedrals;     /* [n][5]: tag_i..tag_l, type                 */
} beads_system_desc;

/* Force field of one replica.  Replaces input::ForceFieldSpec
 * (native_spec.hpp:114-125) after the reference's per-style parameter readers
 * (pair/pair_lj.cu:197-231, bond/bond_harmonic.cu, angle/angle_harmonic.cu:
 * 236-253, dihedral/dihedral_harmonic.cu:293-320).  Tables are indexed by
 * 0-based type id; the LJ tables are full symmetric n_types x n_types. */
typedef struct beads_forcefield_desc {
  int32_t n_types;
  const double* lj_epsilon;      /* [n_types * n_types]                        */
  const double* lj_sigma;        /* [n_types * n_types]                        */
  double lj_cutoff;              /* one global cutoff (pair_lj.cu:201-212)     */
  int32_t lj_shift;              /* subtract U(rc)                             */
  int32_t n_bond_types;
  const double* bond_k;          /* U = 0.5 k (r - r0)^2                       */
  const double* bond_r0;
  int32_t n_angle_types;
  const double* angle_k;         /* U = 0.5 k (theta - theta0)^2               */
  const double* angle_theta0_deg;
  int32_t n_dihedral_types;
  const double* dihedral_k;      /* U = k (1 + d cos(n phi))                   */
  const int32_t* dihedral_d;     /* +1 or -1                                   */
  const int32_t* dihedral_n;     /* >= 0                                       */
  int32_t exclusion_distance;    /* 0 = none, else bond-graph distance 1..3    */
} beads_forcefield_desc;

/* Replaces input::NeighborSpec (native_spec.hpp:139-144). */
typedef struct beads_neighbor_desc {
  double cutoff_buffer;          /* skin                                       */
  uint64_t rebuild_check_every;
  uint64_t sort_every_rebuild;
  uint32_t max_neighbors;
} beads_neighbor_desc;

/* Replaces input::DynamicsSpec (native_spec.hpp:133-137). */
typedef struct beads_dynamics_desc {
  double dt;
  int32_t thermostat;            /* 0 none, 1 berendsen                        */
  double temperature;            /* public units (K in nm_kjmol)               */
  double tau;
} beads_dynamics_desc;

/* Observables of the most recent force evaluation of one replica, the values
 * of one thermo row (native/src/simulation/output/thermo/thermo_output.cu:
 * 437-470).  Totals are reduced in 64-bit fixed point on the device. */
typedef struct beads_observables {
  uint64_t step;
  double pair_pe;
  double bond_pe;
  double angle_pe;
  double dihedral_pe;
  double pe;                     /* sum of the four                            */
  double ke;                     /* after the Berendsen scaling of that step   */
  double virial;                 /* global scalar virial  sum r.F              */
  double temp;                   /* 2 KE / (dof kB), dof = 3N - 3              */
  double press;                  /* s (2 KE + W) / (3 V)                       */
  uint64_t neighbor_build_count;
  uint64_t dangerous_rebuild_count;
} beads_observables;

typedef struct beads_ctx beads_ctx;

/* Interrupt hook: called from the run loop every `every` steps (the
 * reference polls PyErr_CheckSignals every max(1, 100000/N) steps,
 * simulation_run.cpp:92); return non-zero to stop with
 * BEADS_ERR_INTERRUPTED. */
typedef int (*beads_interrupt_fn)(void* user);

/* Whole-run description used by beads_execute(); replaces
 * input::SimulationSpec (native_spec.hpp:169-176) together with its
 * OutputSpec (native_spec.hpp:146-167). */
typedef struct beads_run_desc {
  const beads_system_desc* system;
  const beads_forcefield_desc* forcefield;
  const beads_neighbor_desc* neighbor;
  const beads_dynamics_desc* dynamics;
  uint64_t runsteps;
  uint64_t thermo_every;         /* 0 = no thermo output                       */
  const char* thermo_prefix;
  uint64_t trajectory_every;     /* 0 = no trajectory output                   */
  const char* trajectory_prefix;
  uint32_t trajectory_fields;    /* BEADS_FIELD_* mask, tag always set         */
  const char* final_state_prefix;/* NULL = no final state                      */
  int32_t log_echo;              /* BEADS_ECHO_*                               */
  const char* log_prefix;        /* required for LOG / BOTH                    */
  const char* thermostat_name;   /* "none" or "berendsen" (log only)           */
  const char* exclusion_policy;  /* "none" / "default" / "explicit" (log only) */
  beads_interrupt_fn interrupt;  /* may be NULL                                */
  void* interrupt_user;
} beads_run_desc;

/* ---- build information ---------------------------------------------------
 * Replaces _native.build_info() (native/src/bindings/module.cpp:15-27).
 * Writes a JSON object with the keys real_precision, real_dtype, type_dtype,
 * index_dtype, image_dtype, runstep_dtype into buf (NUL-terminated). */
BEADS_API int beads_build_info(char* buf, size_t buf_size);

/* Message of the last failure on this thread (NUL-terminated, truncated). */
BEADS_API int beads_last_error(char* buf, size_t buf_size);

/* ---- whole simulation with file outputs ----------------------------------
 * Replaces _native.execute_simulation(spec) (module.cpp:36-44 ->
 * SimulationRun(spec).execute(), simulation_run.cpp:237-244): validates,
 * runs `runsteps` velocity-Verlet steps (or a zero-step evaluation), and
 * writes the thermo CSV, binary trajectory, final-state snapshot and log in
 * the reference's formats. */
BEADS_API int beads_execute(const beads_run_desc* run);

/* ---- engine contexts ------------------------------------------------------
 * A context owns the device state of n_replicas independent replicas packed
 * into one set of arrays; every kernel runs over all replicas at once.
 * beads_ctx_create is the one-replica case of beads_batch_create.  Replaces the
 * construction in SimulationRun::SimulationRun (simulation_run.cpp:60-98). */
BEADS_API int beads_ctx_create(const beads_system_desc* system,
                     const beads_forcefield_desc* forcefield,
                     const beads_neighbor_desc* neighbor,
                     const beads_dynamics_desc* dynamics,
                     beads_ctx** out);
BEADS_API int beads_batch_create(uint32_t n_replicas,
                       const beads_system_desc* systems,
                       const beads_forcefield_desc* forcefields,
                       const beads_neighbor_desc* neighbors,
                       const beads_dynamics_desc* dynamics,
                       beads_ctx** out);
BEADS_API void beads_ctx_destroy(beads_ctx* ctx);

/* Neighbour build + force/energy/virial evaluation at the current positions
 * (the reference's initialize_force_state, simulation_run.cpp:113-119, and
 * its zero-step run, :158-172).  Fills one beads_observables per replica. */
BEADS_API int beads_eval(beads_ctx* ctx, beads_observables* out);

/* Advance every replica by `steps` velocity-Verlet steps (the reference's
 * advance_dynamics_step loop, simulation_run.cpp:189-235).  If
 * obs_every > 0, observables are evaluated on steps that are multiples of
 * obs_every; `out` (may be NULL) receives the observables of the last step if
 * it was such a step.  The step loop between output steps is replayed as a
 * CUDA graph; neighbour rebuilds are decided on the device. */
BEADS_API int beads_run(beads_ctx* ctx, uint64_t steps, uint64_t obs_every,
              beads_observables* out);

/* Copy the state of one replica to host arrays in TAG order.  Any pointer may
 * be NULL.  forces are those of the last evaluation. */
BEADS_API int beads_get_state(beads_ctx* ctx, uint32_t replica, float* positions,
                    float* velocities, float* forces, int32_t* images);
/* Overwrite positions/velocities (TAG order, may be NULL) of one replica;
 * positions must be inside the box.  The next step rebuilds the list. */
BEADS_API int beads_set_state(beads_ctx* ctx, uint32_t replica, const float* positions,
                    const float* velocities);

/* Whole-batch host transfers in TAG order, replica after replica (replica r's
 * block starts at the sum of the previous replicas' particle counts).  These
 * are one H2D / D2H copy each plus a device scatter/gather, used by callers
 * that stream the state every call.  Both return once their copies are
 * complete, so the host buffers (pinned or not) may be reused at once.  Any
 * pointer may be NULL. */
BEADS_API int beads_upload_all(beads_ctx* ctx, const float* positions,
                     const float* velocities);
BEADS_API int beads_download_all(beads_ctx* ctx, float* positions, float* velocities);

/* Device-resident views for in-process callers (the autograd wrapper, the
 * benchmark): number of replicas / particles, and the CUDA stream the engine
 * launches on. */
BEADS_API int beads_ctx_info(beads_ctx* ctx, uint32_t* n_replicas,
                   uint64_t* n_particles_total, void** stream);

/* Times `reps` back-to-back launches of one stage on the engine's stream
 * with CUDA events (synchronized on both sides) and returns the mean duration
 * per launch in milliseconds.  stage 0: pair + bonded forces on the current
 * list (no observables); 1: one full MD step; 2: one forced neighbour
 * rebuild; 3: the force kernels as a step launches them (with the second
 * half-kick and the kinetic-energy total), velocities and per-replica step
 * state restored afterwards; 4: the pair-force kernel alone; 5: the bonded
 * kernel alone (forces re-evaluated in full after stages 4 and 5).  Stages 1
 * and 2 advance or rebuild the state they time. */
BEADS_API int beads_profile(beads_ctx* ctx, int32_t stage, uint32_t reps,
                            double* avg_ms);
/* Neighbour-list statistics of the last build over all replicas: total list
 * entries and the largest per-particle count. */
BEADS_API int beads_list_stats(beads_ctx* ctx, uint64_t* total_entries,
                               uint32_t* max_count);

/* Kernel schedule of a context, as five int32 values:
 *   schedule[0] threads per particle of the pair-force kernel: 1, 2 or 4
 *   schedule[1] second half-kick inside the last force kernel (1) or as its
 *               own kernel (0)
 *   schedule[2] batch depth: neighbour-list entries in flight per thread, 4/8
 *   schedule[3] neighbour-list loads bypass L1 (1) or stream through it (0)
 *   schedule[4] (get only) 1 if the autotuner chose the schedule
 * The choice never changes a result (forces are summed in one canonical
 * order).  By default the first beads_run() times the candidates on the
 * context's own batch and keeps the fastest; beads_set_tuning() with
 * schedule[0] = 1, 2 or 4 fixes the schedule (entries 0-3 read), 0 returns it
 * to the autotuner.  No reference counterpart (the reference has one fixed
 * launch shape per kernel). */
BEADS_API int beads_set_tuning(beads_ctx* ctx, const int32_t* schedule);
BEADS_API int beads_get_tuning(beads_ctx* ctx, int32_t* schedule);

/* Neighbour-list layout of a context.  Staged (1, the default when some
 * replica has >= 4 cells on every axis): list rows in the cell order of the
 * last build, and for every group of 128 rows whose stage fits, entries that
 * index a shared-memory copy of the group's stencil cells, from which the
 * pair-force kernel reads every neighbour position.  Slot layout (0): rows
 * and entries by slot, positions gathered from global memory.  The choice
 * never changes a result; switching rebuilds the list before the next force
 * evaluation.  Without a call the autotuner times both layouts at the first
 * run and keeps the faster; after a call it keeps the layout set here.
 * beads_get_list_layout reports 0 when no replica can stage.
 * No reference counterpart (the reference keeps one slot-major list,
 * neighbor_list.cuh:12-71). */
BEADS_API int beads_set_list_layout(beads_ctx* ctx, int32_t staged);
BEADS_API int beads_get_list_layout(beads_ctx* ctx, int32_t* staged);

/* ---- differentiation (no reference counterpart) ------------------------- */
/* Replaces one replica's LJ tables (symmetric [n_types * n_types], same
 * meaning as beads_forcefield_desc.lj_epsilon / lj_sigma); the cutoff and
 * shift setting stay.  The next step re-evaluates forces. */
BEADS_API int beads_set_lj(beads_ctx* ctx, uint32_t replica, const double* epsilon,
                           const double* sigma);
/* Runs `steps` MD steps from the current state (list and forces rebuilt
 * first) keeping a checkpoint of the full step state every
 * `checkpoint_every` steps (0: keep the state of every step, 32 bytes per
 * particle and step, so the backward pass needs no replay), and writes the
 * observables of steps
 * record_from..steps: observables[((step - record_from) * n_replicas + r) * 3
 * + {0, 1, 2}] = potential energy, virial (sum r.F), kinetic energy (as a
 * thermo row reports them).  Up to 4 particle types and 8 bonded types of
 * each kind per replica.  Slots are not reordered during the run. */
BEADS_API int beads_adjoint_forward(beads_ctx* ctx, uint64_t steps, uint64_t record_from,
                                    uint32_t checkpoint_every, double* observables);
/* Reverse pass of the last beads_adjoint_forward(): given dL/d(observables)
 * in the same layout, writes dL/d(epsilon) and dL/d(sigma) per replica and
 * ordered type pair ([r][n_types * n_types], concatenated over replicas in
 * order, each replica with its own n_types) and dL/d(initial positions),
 * dL/d(initial velocities) in tag order ([n_particles_total][3]).  The
 * segments between checkpoints are replayed with the neighbour list of each
 * forward step frozen; afterwards the context is in its end-of-forward
 * state. */
BEADS_API int beads_adjoint_backward(beads_ctx* ctx, const double* observables_grad,
                                     double* grad_epsilon, double* grad_sigma,
                                     float* grad_positions, float* grad_velocities);

/* Replaces one replica's harmonic bonded parameters, per local type (NULL
 * arrays leave that parameter unchanged; theta0 in degrees). */
BEADS_API int beads_set_bonded(beads_ctx* ctx, uint32_t replica, const double* bond_k,
                               const double* bond_r0, const double* angle_k,
                               const double* angle_theta0_deg, const double* dihedral_k);
/* Bonded parameter gradients of the last beads_adjoint_backward(), by global
 * type (every replica's types in batch order): grad_bond [types][2] = d/dk,
 * d/dr0; grad_angle [types][2] = d/dk, d/dtheta0 (per degree); grad_dihedral
 * [types] = d/dk.  NULL pointers are skipped. */
BEADS_API int beads_adjoint_bonded_grads(beads_ctx* ctx, double* grad_bond, double* grad_angle,
                                         double* grad_dihedral);

/* Device counters of one replica, without stepping it: counters[0] completed
 * MD steps, [1] neighbour builds, [2] dangerous rebuilds (the quantities the
 * reference's run log reports, log_output.cpp:370-404), [3] launches of the
 * rebuild chain so far for the whole context (a captured step launches the
 * chain only when some replica rebuilds).  counters has 4 entries. */
BEADS_API int beads_counters(beads_ctx* ctx, uint32_t replica, uint64_t* counters);

/* Kernel launches of the current schedule: *per_step kernels every MD step
 * launches, and *per_rebuild_chain kernels each time the rebuild chain runs
 * (counters[3] of beads_counters counts those runs).  *per_rebuild_chain is 0
 * when every step launches the chain itself (no conditional graph node, or
 * graphs switched off with BEADS_GRAPHS=0); *per_step then includes it.
 * Counted as the kernel nodes of one captured step; nothing runs.  No
 * counterpart in the reference (measurement). */
BEADS_API int beads_launch_counts(beads_ctx* ctx, uint32_t* per_step,
                                  uint32_t* per_rebuild_chain);

/* Steepest descent with a per-particle displacement cap, used to relax
 * random initial configurations: x += dmax * F / max(|F|, fref), with the LJ
 * force evaluated on r^2 clamped to >= (0.7 sigma)^2 so overlaps stay finite.
 * Not a reference feature (the reference has no minimiser). */
BEADS_API int beads_minimize(beads_ctx* ctx, uint32_t iterations, float dmax,
                   float fref);

/* ---- allocation-free cell sort ------------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * host codes that own all device memory through their own pool, and step
 * loops that must not synchronize the device (cudaMalloc/cudaFree do).  Bins
 * n particles (device positions [n][3], float) into the cell grid the
 * neighbour build uses for this box and rc + skin (same plan and cell-id
 * rules), then sorts them stably by cell: d_cell_of[i] = cell of particle i,
 * d_order = particle indices grouped by cell (ascending inside a cell),
 * d_cell_start[c] = first entry of cell c in d_order (n_cells + 1 entries;
 * *n_cells_out receives n_cells).  All device buffers are the caller's; the
 * per-cell counters live in a static device array of BEADS_STATIC_MAX_CELLS
 * cells that every GPU loading the library holds until exit, so grids with
 * more cells are rejected with BEADS_ERR_INVALID.  Work is enqueued on
 * `stream` (a cudaStream_t, NULL = legacy default stream) and is complete
 * when that stream is.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) and should come before any stream
 * capture.  All calls share the array, so calls that overlap on the GPU
 * (different streams or host threads without ordering) race. */
#define BEADS_STATIC_MAX_CELLS 65536u
BEADS_API int beads_cell_sort_static(const float* d_positions, uint32_t n,
                                     const float box_lo[3], const float box_hi[3],
                                     double cutoff, double skin, uint32_t* d_cell_of,
                                     uint32_t* d_order, uint32_t* d_cell_start,
                                     uint32_t cell_start_capacity,
                                     uint32_t* n_cells_out, void* stream);

/* ---- parity / debugging views (TAG order) --------------------------------
 * Cell id of every particle from the last neighbour build (the reference's
 * particle_cell, cell_list_build.cu:135-166). */
BEADS_API int beads_debug_cells(beads_ctx* ctx, uint32_t replica, uint32_t* cell_by_tag);
/* Full neighbour list of the last build: counts[tag-1] and the partner tags
 * in partners[(tag-1) * cap + k].  Replaces the reference's NeighborList
 * storage (neighbor_list.cuh:12-71) as a host view. */
BEADS_API int beads_debug_neighbors(beads_ctx* ctx, uint32_t replica, uint32_t cap,
                          uint32_t* counts, uint32_t* partners);
/* Neighbour-build path of a replica: 0 direct, 1 regular_cell,
 * 2 small_dimension (neighbor_plan.cpp:107-128) and its cell grid. */
BEADS_API int beads_debug_plan(beads_ctx* ctx, uint32_t replica, int32_t* path,
                     uint32_t* ncells3);

#ifdef __cplusplus
}
#endif

#endif /* BEADS_B200_H */
