// ref_neighbors.cu -- dumps the reference engine's OWN neighbour list.
//
// TEST INFRASTRUCTURE ONLY (a checker): nothing in beads_b200 loads it.  It is
// compiled by oracle/build_ref.py against the reference's headers and linked
// with the reference's own object files (the same objects as its _native
// module, minus that module's PYBIND11_MODULE translation unit), so the list it
// returns is the one the reference's engine builds, not a restatement.
//
// What it drives (paths inside the reference project):
//   spec dict -> input::SimulationSpec   native/src/bindings/native_spec_parser.cpp:755-790
//   host / device state, force field     native/src/simulation/simulation_run.cpp:60-98
//   NeighborSystem::initialize_for_run   native/src/simulation/neighbor/neighbor_system.cpp:71-77
//   list storage (slot-major)            native/src/simulation/neighbor/neighbor_list.cuh:12-71
//
// neighbor_dump(spec) performs the initial build exactly as a run does before
// its first force evaluation, then returns, in TAG order (tag t at row t - 1):
// counts[n] (clamped to max_neighbors as the reference stores them), the
// partner tags partners[n][max_neighbors] (row-major, 0 past the count), the
// overflow flag, the build path name and the excluded-pair count.  (The
// reference keeps its cell grid private, so cell ids are not returned.)
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "bindings/native_spec_parser.hpp"
#include "forcefield/force_field_model.hpp"
#include "simulation/neighbor/neighbor_system.hpp"
#include "system/state/device_state.cuh"
#include "system/state/host_state.hpp"

namespace py = pybind11;

namespace {

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
std::vector<T> download(const T* device, size_t n) {
  std::vector<T> host(n);
  if (n) check(cudaMemcpy(host.data(), device, n * sizeof(T), cudaMemcpyDeviceToHost), "copy");
  return host;
}

py::dict neighbor_dump(const py::object& spec_obj) {
  using namespace beads;
  const input::SimulationSpec spec = bindings::parse_native_spec(spec_obj);
  system::state::HostState host(spec.system);
  forcefield::ForceFieldModel forcefield(spec.forcefield, host);
  system::state::DeviceState device(host);
  simulation::neighbor::NeighborSystem neighbors(
      spec.neighbor, forcefield.max_cutoff(), host, forcefield.requires_tag_to_slot_map(),
      spec.forcefield.bonded_exclusion_distance);
  int overflow = 0;
  try {
    neighbors.initialize_for_run(device.particles(), host.box(), nullptr);
  } catch (const std::exception&) {
    overflow = 1;  // the reference throws after an overflowing build
  }
  check(cudaDeviceSynchronize(), "sync");

  const auto view = neighbors.neighbor_list().view();
  const size_t n = view.n_particles, cap = view.max_neighbors;
  const auto count = download(view.neighbor_count, n);
  const auto index = download(view.neighbor_index, n * cap);
  const auto tag = download(device.particles().tag().data(), n);

  py::array_t<uint32_t> counts(std::vector<py::ssize_t>{static_cast<py::ssize_t>(n)});
  py::array_t<uint32_t> partners(
      std::vector<py::ssize_t>{static_cast<py::ssize_t>(n), static_cast<py::ssize_t>(cap)});
  auto c = counts.mutable_unchecked<1>();
  auto p = partners.mutable_unchecked<2>();
  for (size_t i = 0; i < n; ++i) {
    c(i) = 0;
    for (size_t k = 0; k < cap; ++k) p(i, k) = 0;
  }
  for (size_t slot = 0; slot < n; ++slot) {
    const size_t row = tag[slot] - 1;  // tags are 1-based
    const uint32_t m = count[slot] < cap ? count[slot] : static_cast<uint32_t>(cap);
    c(row) = count[slot];
    for (uint32_t k = 0; k < m; ++k) {
      // neighbor_index_slot(k, n, slot) = k * n + slot (neighbor_list.cuh:12-19)
      p(row, k) = tag[index[k * n + slot]];
    }
  }
  py::dict out;
  out["counts"] = counts;
  out["partners"] = partners;
  out["overflow"] = overflow;
  out["path"] = std::string(neighbors.path_name());
  out["excluded_pairs"] = static_cast<uint64_t>(neighbors.excluded_pair_count());
  out["builds"] = static_cast<uint64_t>(neighbors.build_count());
  return out;
}

}  // namespace

PYBIND11_MODULE(_ref_neighbors, m) {
  m.doc() = "Checker: the reference engine's own neighbour list after the initial build";
  m.def("neighbor_dump", &neighbor_dump);
}
