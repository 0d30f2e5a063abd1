// outputs.hpp -- file outputs in the reference's formats.
//   thermo CSV      native/src/simulation/output/thermo/thermo_output.cu:470-507
//   trajectory      native/src/simulation/output/trajectory/trajectory_output.cu:32-45, 144-170, 555-596
//   final state     native/src/simulation/output/snapshot/final_state_output.cu:110-185
//   log             native/src/simulation/output/log/log_output.cpp:17-404
#pragma once

#include <cstdint>
#include <fstream>
#include <string>
#include <vector>

#include "engine.hpp"

namespace bb {

struct ThermoSchema {
  bool bond = false, angle = false, dihedral = false;
};

class ThermoCsv {
 public:
  ThermoCsv(const std::string& prefix, ThermoSchema schema);
  void write(const beads_observables& o);
  void flush();

 private:
  std::ofstream out_;
  std::string path_;
  ThermoSchema schema_;
};

class TrajectoryFile {
 public:
  TrajectoryFile(const std::string& prefix, uint32_t field_mask, const char* units,
                 uint64_t n_particles);
  void write_frame(uint64_t step, const float lo[3], const float hi[3],
                   const Engine::SlotView& sv, const std::vector<int32_t>& type_by_tag);
  void flush();
  static uint64_t record_bytes(uint32_t mask);

 private:
  std::ofstream out_;
  std::string path_;
  uint32_t mask_;
  uint64_t n_;
};

void write_final_state(const std::string& prefix, const char* units, uint64_t step,
                       const float lo[3], const float hi[3], const Engine::SlotView& sv,
                       const std::vector<int32_t>& type_by_tag);

class LogSink {
 public:
  LogSink(int echo, const char* prefix);
  bool active() const { return screen_ || file_; }
  void message(const char* level, const std::string& text);
  void thermo_row(const beads_observables& o, ThermoSchema schema);
  void flush();

 private:
  bool screen_ = false, file_ = false, wrote_ = false, header_ = false;
  std::ofstream out_;
  std::string path_;
};

std::string log_label(const std::string& label, const std::string& value);

}  // namespace bb
