// capi.cpp -- the extern "C" boundary declared in include/beads_b200.h.
#include <algorithm>
#include <chrono>
#include <memory>
#include <cstring>
#include <functional>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "engine.hpp"
#include "outputs.hpp"
#include "trace.hpp"

struct beads_ctx {
  bb::Engine* engine = nullptr;
};

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& message) {
  g_last_error = message;
  return code;
}

template <typename F>
int guarded(F&& body) {
  try {
    body();
    g_last_error.clear();
    return BEADS_OK;
  } catch (const bb::InvalidArgument& e) {
    return fail(BEADS_ERR_INVALID, e.what());
  } catch (const std::invalid_argument& e) {
    return fail(BEADS_ERR_INVALID, e.what());
  } catch (const bb::NeighborOverflow& e) {
    return fail(BEADS_ERR_NEIGHBOR_OVERFLOW, e.what());
  } catch (const bb::NonFinite& e) {
    return fail(BEADS_ERR_NONFINITE, e.what());
  } catch (const bb::CudaError& e) {
    return fail(BEADS_ERR_CUDA, e.what());
  } catch (const std::overflow_error& e) {
    return fail(BEADS_ERR_OVERFLOW, e.what());
  } catch (const std::bad_alloc&) {
    return fail(BEADS_ERR_RUNTIME, "host allocation failed.");
  } catch (const std::exception& e) {
    const std::string what = e.what();
    if (what == "interrupted") return fail(BEADS_ERR_INTERRUPTED, "interrupted");
    return fail(BEADS_ERR_RUNTIME, what);
  }
}

void require(bool cond, const char* message) {
  if (!cond) throw bb::InvalidArgument(message);
}

const char* units_name(int units) { return units == BEADS_UNITS_NM_KJMOL ? "nm_kjmol" : "reduced"; }

std::string real3(const float v[3]) {
  std::ostringstream s;
  s << '(' << v[0] << ',' << v[1] << ',' << v[2] << ')';
  return s.str();
}

template <typename T>
std::string str(const T& v) {
  std::ostringstream s;
  s << v;
  return s.str();
}

// The whole run of one simulation spec, with file outputs, following the
// reference's SimulationRun (native/src/simulation/simulation_run.cpp:
// 113-244): initial build + forces (step 0 outputs), then runsteps steps with
// outputs on multiples of each output's `every`, then the final state.
void execute_run(const beads_run_desc& run) {
  bb::TraceRange trace("beads.execute");
  require(run.system && run.forcefield && run.neighbor && run.dynamics,
          "run description is incomplete.");
  const beads_system_desc& sys = *run.system;
  bb::Engine engine(1, run.system, run.forcefield, run.neighbor, run.dynamics);
  const bb::ReplicaHost& h = engine.replica(0);
  const char* units = units_name(sys.units);

  bb::ThermoSchema schema;
  schema.bond = sys.n_bonds > 0;
  schema.angle = sys.n_angles > 0;
  schema.dihedral = sys.n_dihedrals > 0;
  std::vector<int32_t> type_by_tag(sys.n_particles);
  for (uint32_t k = 0; k < sys.n_particles; ++k) {
    type_by_tag[(sys.tags ? sys.tags[k] : k + 1) - 1] = sys.types[k];
  }

  const bool thermo = run.thermo_every > 0;
  const bool traj = run.trajectory_every > 0;
  const bool final_state = run.final_state_prefix != nullptr;
  bb::LogSink log(run.log_echo, run.log_prefix);
  const bool any_output = thermo || traj || final_state || log.active();
  if (run.runsteps == 0 && !any_output) return;

  std::unique_ptr<bb::ThermoCsv> csv;
  std::unique_ptr<bb::TrajectoryFile> trj;
  if (thermo) csv.reset(new bb::ThermoCsv(run.thermo_prefix ? run.thermo_prefix : "", schema));
  if (traj) {
    trj.reset(new bb::TrajectoryFile(run.trajectory_prefix ? run.trajectory_prefix : "",
                                     run.trajectory_fields, units, sys.n_particles));
  }

  const auto t0 = std::chrono::steady_clock::now();
  if (log.active()) {
    std::ostringstream m;
    m << "execute start\n" << bb::log_label("units", units) << '\n'
      << bb::log_label("particles", str(sys.n_particles)) << '\n'
      << bb::log_label("box_lo", real3(sys.box_lo)) << '\n'
      << bb::log_label("box_hi", real3(sys.box_hi)) << '\n';
    float len[3] = {sys.box_hi[0] - sys.box_lo[0], sys.box_hi[1] - sys.box_lo[1],
                    sys.box_hi[2] - sys.box_lo[2]};
    m << bb::log_label("box_lengths", real3(len)) << '\n'
      << bb::log_label("runsteps", str(run.runsteps));
    log.message("INFO", m.str());
    std::ostringstream dt_text;
    dt_text << std::setprecision(9) << static_cast<float>(run.dynamics->dt);
    std::ostringstream d;
    d << "dynamics summary\n" << bb::log_label("style", "velocity_verlet") << '\n'
      << bb::log_label("dt", dt_text.str()) << '\n'
      << bb::log_label("thermostat", run.thermostat_name ? run.thermostat_name : "none");
    log.message("INFO", d.str());
    std::ostringstream nmsg;
    nmsg << "neighbor summary\n" << bb::log_label("cutoff_buffer", str(static_cast<float>(run.neighbor->cutoff_buffer))) << '\n'
         << bb::log_label("path", bb::path_name(h.plan.path)) << '\n'
         << bb::log_label("rebuild_check_every", str(run.neighbor->rebuild_check_every)) << '\n'
         << bb::log_label("sort_every_rebuild", str(run.neighbor->sort_every_rebuild)) << '\n'
         << bb::log_label("max_neighbors", str(run.neighbor->max_neighbors));
    log.message("INFO", nmsg.str());
    std::ostringstream f;
    f << "forcefield summary\n" << bb::log_label("pair", "lj") << '\n'
      << bb::log_label("bond", schema.bond ? "harmonic" : "none") << '\n'
      << bb::log_label("angle", schema.angle ? "harmonic" : "none") << '\n'
      << bb::log_label("dihedral", schema.dihedral ? "harmonic" : "none") << '\n'
      << bb::log_label("bonded_exclusion_policy", run.exclusion_policy ? run.exclusion_policy : "none") << '\n'
      << bb::log_label("bonded_exclusion_distance",
                       run.forcefield->exclusion_distance > 0 ? str(run.forcefield->exclusion_distance) : "none")
      << '\n' << bb::log_label("bonded_excluded_pairs", str(h.excluded_pairs));
    log.message("INFO", f.str());
    std::ostringstream t;
    t << "topology summary\n" << bb::log_label("bonds", str(sys.n_bonds)) << '\n'
      << bb::log_label("angles", str(sys.n_angles)) << '\n'
      << bb::log_label("dihedrals", str(sys.n_dihedrals));
    log.message("INFO", t.str());
    static const char* echo_names[] = {"none", "screen", "log", "both"};
    std::ostringstream o;
    o << "output summary\n" << bb::log_label("thermo", thermo ? "enabled" : "disabled") << '\n'
      << bb::log_label("final_state", final_state ? "enabled" : "disabled") << '\n'
      << bb::log_label("trajectory", traj ? "enabled" : "disabled") << '\n'
      << bb::log_label("log", echo_names[run.log_echo & 3]);
    log.message("INFO", o.str());
  }

  std::vector<beads_observables> obs;
  bb::Engine::SlotView sv;
  auto emit = [&](uint64_t step, bool have_obs) {
    if (thermo && step % run.thermo_every == 0) {
      if (!have_obs) throw std::logic_error("thermo step without observables.");
      engine.observables(obs);
      csv->write(obs[0]);
      log.thermo_row(obs[0], schema);
    }
    if (traj && step % run.trajectory_every == 0) {
      engine.slot_view(0, sv);
      trj->write_frame(step, h.box_lo, h.box_hi, sv, type_by_tag);
    }
  };

  engine.eval();
  emit(0, true);
  // The reference polls for an interrupt every max(1, 100000 / N) steps
  // (simulation_run.cpp:92); here the poll runs at the first chunk boundary
  // (chunks hold at most 16 steps) at or after each such interval, inside
  // Engine::run, and once before the final outputs.
  const uint64_t check_interval = std::max<uint64_t>(1, 100000 / std::max<uint32_t>(1, sys.n_particles));
  std::function<bool()> poll;
  if (run.interrupt) poll = [&] { return run.interrupt(run.interrupt_user) != 0; };
  while (engine.step() < run.runsteps) {
    const uint64_t s = engine.step();
    uint64_t next = run.runsteps;
    if (thermo) next = std::min(next, (s / run.thermo_every + 1) * run.thermo_every);
    if (traj) next = std::min(next, (s / run.trajectory_every + 1) * run.trajectory_every);
    const uint64_t target = next;
    const bool obs_at_target = thermo && target % run.thermo_every == 0;
    engine.run(target - s, obs_at_target ? target : 0, run.interrupt ? &poll : nullptr,
               check_interval);
    emit(target, obs_at_target);
    if (run.interrupt && engine.step() < run.runsteps && poll()) {
      throw std::runtime_error("interrupted");
    }
  }
  if (run.interrupt && run.runsteps > 0 && poll()) {
    throw std::runtime_error("interrupted");
  }
  if (final_state) {
    engine.slot_view(0, sv);
    bb::write_final_state(run.final_state_prefix, units, engine.step(), h.box_lo, h.box_hi, sv,
                          type_by_tag);
  }
  engine.check_status();
  const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (csv) csv->flush();
  if (trj) trj->flush();
  if (log.active()) {
    engine.observables(obs);
    std::ostringstream e;
    e << "execute end\n" << bb::log_label("runsteps", str(run.runsteps)) << '\n';
    std::ostringstream w;
    w << std::setprecision(9) << wall;
    e << bb::log_label("run_wall_s", w.str()) << '\n';
    if (run.runsteps) {
      std::ostringstream sps;
      sps << std::setprecision(9) << static_cast<double>(run.runsteps) / wall;
      e << bb::log_label("steps_per_second", sps.str()) << '\n';
    } else {
      e << bb::log_label("steps_per_second", "not_applicable") << '\n';
    }
    e << bb::log_label("neighbor_build_count", str(obs[0].neighbor_build_count)) << '\n'
      << bb::log_label("dangerous_rebuild_count", str(obs[0].dangerous_rebuild_count));
    log.message("INFO", e.str());
    log.flush();
  }
}

}  // namespace

namespace bb {
void set_last_error(const char* message) { g_last_error = message; }
}  // namespace bb

extern "C" {

int beads_build_info(char* buf, size_t buf_size) {
  static const char kInfo[] =
      "{\"real_precision\": \"single\", \"real_dtype\": \"float32\", "
      "\"type_dtype\": \"int32\", \"index_dtype\": \"uint32\", "
      "\"image_dtype\": \"int32\", \"runstep_dtype\": \"uint64\"}";
  if (!buf || buf_size < sizeof(kInfo)) return fail(BEADS_ERR_INVALID, "buffer too small");
  std::memcpy(buf, kInfo, sizeof(kInfo));
  return BEADS_OK;
}

int beads_last_error(char* buf, size_t buf_size) {
  if (!buf || buf_size == 0) return BEADS_ERR_INVALID;
  const size_t n = std::min(buf_size - 1, g_last_error.size());
  std::memcpy(buf, g_last_error.data(), n);
  buf[n] = '\0';
  return BEADS_OK;
}

int beads_execute(const beads_run_desc* run) {
  return guarded([&] {
    require(run != nullptr, "run description is NULL.");
    execute_run(*run);
  });
}

int beads_ctx_create(const beads_system_desc* system, const beads_forcefield_desc* ff,
                     const beads_neighbor_desc* nbr, const beads_dynamics_desc* dyn,
                     beads_ctx** out) {
  return beads_batch_create(1, system, ff, nbr, dyn, out);
}

int beads_batch_create(uint32_t n, const beads_system_desc* systems,
                       const beads_forcefield_desc* ffs, const beads_neighbor_desc* nbrs,
                       const beads_dynamics_desc* dyns, beads_ctx** out) {
  return guarded([&] {
    require(out && systems && ffs && nbrs && dyns, "NULL argument.");
    *out = nullptr;
    auto* c = new beads_ctx;
    try {
      c->engine = new bb::Engine(n, systems, ffs, nbrs, dyns);
    } catch (...) {
      delete c;
      throw;
    }
    *out = c;
  });
}

void beads_ctx_destroy(beads_ctx* ctx) {
  if (!ctx) return;
  delete ctx->engine;
  delete ctx;
}

int beads_eval(beads_ctx* ctx, beads_observables* out) {
  return guarded([&] {
    require(ctx && ctx->engine, "NULL context.");
    ctx->engine->eval();
    if (out) {
      std::vector<beads_observables> o;
      ctx->engine->observables(o);
      std::memcpy(out, o.data(), o.size() * sizeof(beads_observables));
    }
  });
}

int beads_run(beads_ctx* ctx, uint64_t steps, uint64_t obs_every, beads_observables* out) {
  return guarded([&] {
    require(ctx && ctx->engine, "NULL context.");
    const bool obs = ctx->engine->run(steps, obs_every);
    if (out && obs) {
      std::vector<beads_observables> o;
      ctx->engine->observables(o);
      std::memcpy(out, o.data(), o.size() * sizeof(beads_observables));
    }
  });
}

int beads_get_state(beads_ctx* ctx, uint32_t replica, float* positions, float* velocities,
                    float* forces, int32_t* images) {
  return guarded([&] {
    require(ctx && ctx->engine, "NULL context.");
    require(replica < ctx->engine->n_replicas(), "replica index out of range.");
    ctx->engine->state(replica, positions, velocities, forces, images);
  });
}

int beads_set_state(beads_ctx* ctx, uint32_t replica, const float* positions,
                    const float* velocities) {
  return guarded([&] {
    require(ctx && ctx->engine, "NULL context.");
    require(replica < ctx->engine->n_replicas(), "replica index out of range.");
    ctx->engine->set_state(replica, positions, velocities);
  });
}

int beads_upload_all(beads_ctx* ctx, const float* positions, const float* velocities) {
  return guarded([&] {
    require(ctx && ctx->engine, "NULL context.");
    ctx->engine->upload_all(positions, velocities);
  });
}

int beads_download_all(beads_ctx* ctx, float* positions, float* velocities) {
  return guarded([&] {
    require(ctx && ctx->engine, "NULL context.");
    ctx->engine->download_all(positions, velocities);
  });
}

int beads_ctx_info(beads_ctx* ctx, uint32_t* n_replicas, uint64_t* n_particles_total,
                   void** stream) {
  return guarded([&] {
    require(ctx && ctx->engine, "NULL context.");
    if (n_replicas) *n_replicas = ctx->engine->n_replicas();
    if (n_particles_total) *n_particles_total = ctx->engine->n_particles_total();
    if (stream) *stream = reinterpret_cast<void*>(ctx->engine->stream());
  });
}

int beads_minimize(beads_ctx* ctx, uint32_t iterations, float dmax, float fref) {
  return guarded([&] {
    require(ctx && ctx->engine, "NULL context.");
    require(dmax > 0.f && fref > 0.f, "minimize needs positive dmax and fref.");
    ctx->engine->minimize(iterations, dmax, fref);
  });
}

int beads_profile(beads_ctx* ctx, int32_t stage, uint32_t reps, double* avg_ms) {
  return guarded([&] {
    require(ctx && ctx->engine && avg_ms, "NULL argument.");
    *avg_ms = ctx->engine->profile(stage, reps);
  });
}

int beads_list_stats(beads_ctx* ctx, uint64_t* total_entries, uint32_t* max_count) {
  return guarded([&] {
    require(ctx && ctx->engine, "NULL context.");
    ctx->engine->list_stats(total_entries, max_count);
  });
}

int beads_set_tuning(beads_ctx* ctx, const int32_t* schedule) {
  return guarded([&] {
    require(ctx && ctx->engine && schedule, "NULL argument.");
    ctx->engine->set_tuning(schedule[0], schedule[1], schedule[2], schedule[3]);
  });
}

int beads_get_tuning(beads_ctx* ctx, int32_t* schedule) {
  return guarded([&] {
    require(ctx && ctx->engine && schedule, "NULL argument.");
    int t = 0, f = 0, u = 0, nl = 0, a = 0;
    ctx->engine->tuning(&t, &f, &u, &nl, &a);
    schedule[0] = t;
    schedule[1] = f;
    schedule[2] = u;
    schedule[3] = nl;
    schedule[4] = a;
  });
}

int beads_set_list_layout(beads_ctx* ctx, int32_t staged) {
  return guarded([&] {
    require(ctx && ctx->engine, "NULL argument.");
    ctx->engine->set_list_staged(staged != 0);
  });
}

int beads_get_list_layout(beads_ctx* ctx, int32_t* staged) {
  return guarded([&] {
    require(ctx && ctx->engine && staged, "NULL argument.");
    *staged = ctx->engine->list_staged() ? 1 : 0;
  });
}

int beads_set_lj(beads_ctx* ctx, uint32_t replica, const double* epsilon, const double* sigma) {
  return guarded([&] {
    require(ctx && ctx->engine && epsilon && sigma, "NULL argument.");
    require(replica < ctx->engine->n_replicas(), "replica index out of range.");
    ctx->engine->set_lj(replica, epsilon, sigma);
  });
}

int beads_adjoint_forward(beads_ctx* ctx, uint64_t steps, uint64_t record_from,
                          uint32_t checkpoint_every, double* observables) {
  return guarded([&] {
    require(ctx && ctx->engine && observables, "NULL argument.");
    ctx->engine->adjoint_forward(steps, record_from, checkpoint_every, observables);
  });
}

int beads_adjoint_backward(beads_ctx* ctx, const double* observables_grad, double* grad_epsilon,
                           double* grad_sigma, float* grad_positions, float* grad_velocities) {
  return guarded([&] {
    require(ctx && ctx->engine && observables_grad && grad_epsilon && grad_sigma &&
                grad_positions && grad_velocities,
            "NULL argument.");
    ctx->engine->adjoint_backward(observables_grad, grad_epsilon, grad_sigma, grad_positions,
                                  grad_velocities);
  });
}

int beads_set_bonded(beads_ctx* ctx, uint32_t replica, const double* bond_k,
                     const double* bond_r0, const double* angle_k,
                     const double* angle_theta0_deg, const double* dihedral_k) {
  return guarded([&] {
    require(ctx && ctx->engine, "NULL context.");
    require(replica < ctx->engine->n_replicas(), "replica index out of range.");
    ctx->engine->set_bonded(replica, bond_k, bond_r0, angle_k, angle_theta0_deg, dihedral_k);
  });
}

int beads_adjoint_bonded_grads(beads_ctx* ctx, double* grad_bond, double* grad_angle,
                               double* grad_dihedral) {
  return guarded([&] {
    require(ctx && ctx->engine, "NULL context.");
    ctx->engine->adjoint_bonded_grads(grad_bond, grad_angle, grad_dihedral);
  });
}

int beads_counters(beads_ctx* ctx, uint32_t replica, uint64_t* counters) {
  return guarded([&] {
    require(ctx && ctx->engine && counters, "NULL argument.");
    require(replica < ctx->engine->n_replicas(), "replica index out of range.");
    ctx->engine->counters(replica, counters);
  });
}

int beads_launch_counts(beads_ctx* ctx, uint32_t* per_step, uint32_t* per_rebuild_chain) {
  return guarded([&] {
    require(ctx && ctx->engine && per_step && per_rebuild_chain, "NULL argument.");
    ctx->engine->launch_counts(*per_step, *per_rebuild_chain);
  });
}

int beads_debug_cells(beads_ctx* ctx, uint32_t replica, uint32_t* cell_by_tag) {
  return guarded([&] {
    require(ctx && ctx->engine && cell_by_tag, "NULL argument.");
    require(replica < ctx->engine->n_replicas(), "replica index out of range.");
    ctx->engine->debug_cells(replica, cell_by_tag);
  });
}

int beads_debug_neighbors(beads_ctx* ctx, uint32_t replica, uint32_t cap, uint32_t* counts,
                          uint32_t* partners) {
  return guarded([&] {
    require(ctx && ctx->engine && counts && partners, "NULL argument.");
    require(replica < ctx->engine->n_replicas(), "replica index out of range.");
    ctx->engine->debug_neighbors(replica, cap, counts, partners);
  });
}

int beads_debug_plan(beads_ctx* ctx, uint32_t replica, int32_t* path, uint32_t* ncells3) {
  return guarded([&] {
    require(ctx && ctx->engine, "NULL context.");
    require(replica < ctx->engine->n_replicas(), "replica index out of range.");
    const bb::ReplicaHost& h = ctx->engine->replica(replica);
    if (path) *path = static_cast<int32_t>(h.plan.path);
    if (ncells3) {
      for (int a = 0; a < 3; ++a) ncells3[a] = h.plan.nc[a];
    }
  });
}

}  // extern "C"
