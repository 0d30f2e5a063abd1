// outputs.cpp -- writers for the thermo CSV, binary trajectory, final-state
// snapshot and log.  The byte layouts are the reference's file contracts
// (readers in python/beads/io.py and python/beads/_state_snapshot.py consume
// them); the code is this project's own.
#include "outputs.hpp"

#include <cstring>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <stdexcept>

namespace bb {
namespace {

constexpr uint32_t kFormatVersion = 1;
constexpr uint32_t kEndianMarker = 0x01020304u;

template <typename T>
void put(std::ofstream& out, const T& value) {
  out.write(reinterpret_cast<const char*>(&value), sizeof(T));
}

void put_bytes(std::ofstream& out, const void* data, size_t n) {
  if (n) out.write(reinterpret_cast<const char*>(data), static_cast<std::streamsize>(n));
}

void put_units(std::ofstream& out, const char* units) {
  const std::string u(units);
  put<uint64_t>(out, u.size());
  put_bytes(out, u.data(), u.size());
}

// Reals are printed as the engine's float type with 9 significant digits.
std::string real9(double v) {
  std::ostringstream s;
  s << std::setprecision(9) << static_cast<float>(v);
  return s.str();
}

}  // namespace

ThermoCsv::ThermoCsv(const std::string& prefix, ThermoSchema schema)
    : path_(prefix + ".thermo.csv"), schema_(schema) {
  if (prefix.empty()) throw InvalidArgument("output.thermo.prefix must not be empty.");
  out_.open(path_);
  if (!out_) throw std::runtime_error("failed to open thermo output file " + path_ + ".");
  out_ << "step,pe,pair_pe";
  if (schema_.bond) out_ << ",bond_pe";
  if (schema_.angle) out_ << ",angle_pe";
  if (schema_.dihedral) out_ << ",dihedral_pe";
  out_ << ",ke,temp,press\n";
}

void ThermoCsv::write(const beads_observables& o) {
  out_ << o.step << ',' << real9(o.pe) << ',' << real9(o.pair_pe);
  if (schema_.bond) out_ << ',' << real9(o.bond_pe);
  if (schema_.angle) out_ << ',' << real9(o.angle_pe);
  if (schema_.dihedral) out_ << ',' << real9(o.dihedral_pe);
  out_ << ',' << real9(o.ke) << ',' << real9(o.temp) << ',' << real9(o.press) << '\n';
  if (!out_) throw std::runtime_error("failed to write thermo output file " + path_ + ".");
}

void ThermoCsv::flush() { out_.flush(); }

uint64_t TrajectoryFile::record_bytes(uint32_t mask) {
  uint64_t b = 4;  // tag
  if (mask & BEADS_FIELD_TYPE) b += 4;
  if (mask & BEADS_FIELD_POSITION) b += 12;
  if (mask & BEADS_FIELD_IMAGE) b += 12;
  if (mask & BEADS_FIELD_VELOCITY) b += 12;
  if (mask & BEADS_FIELD_FORCE) b += 12;
  return b;
}

TrajectoryFile::TrajectoryFile(const std::string& prefix, uint32_t field_mask,
                               const char* units, uint64_t n_particles)
    : path_(prefix + ".trajectory.beadsbin"), mask_(field_mask | BEADS_FIELD_TAG), n_(n_particles) {
  if (prefix.empty()) throw InvalidArgument("output.trajectory.prefix must not be empty.");
  out_.open(path_, std::ios::binary | std::ios::trunc);
  if (!out_) throw std::runtime_error("failed to open trajectory output file " + path_ + ".");
  const char magic[] = "BEADS_TRAJECTORY";
  put_bytes(out_, magic, sizeof(magic) - 1);
  put<uint32_t>(out_, kFormatVersion);
  put<uint32_t>(out_, kEndianMarker);
  put<uint32_t>(out_, 4);  // real
  put<uint32_t>(out_, 4);  // index
  put<uint32_t>(out_, 4);  // image
  put<uint32_t>(out_, 4);  // type
  put<uint32_t>(out_, 4);  // tag
  put_units(out_, units);
  put<uint32_t>(out_, mask_);
  put<uint64_t>(out_, n_);
  put<uint64_t>(out_, record_bytes(mask_));
}

void TrajectoryFile::write_frame(uint64_t step, const float lo[3], const float hi[3],
                                 const Engine::SlotView& sv,
                                 const std::vector<int32_t>& type_by_tag) {
  put<uint64_t>(out_, step);
  put_bytes(out_, lo, 12);
  put_bytes(out_, hi, 12);
  const uint64_t rb = record_bytes(mask_);
  std::vector<char> buf(rb * sv.tag.size());
  for (size_t k = 0; k < sv.tag.size(); ++k) {
    char* p = buf.data() + k * rb;
    auto w = [&p](const void* src, size_t n) {
      std::memcpy(p, src, n);
      p += n;
    };
    w(&sv.tag[k], 4);
    if (mask_ & BEADS_FIELD_TYPE) w(&type_by_tag[sv.tag[k] - 1], 4);
    if (mask_ & BEADS_FIELD_POSITION) w(&sv.pos[k], 12);
    if (mask_ & BEADS_FIELD_IMAGE) w(&sv.img[k], 12);
    if (mask_ & BEADS_FIELD_VELOCITY) w(&sv.vel[k], 12);
    if (mask_ & BEADS_FIELD_FORCE) w(&sv.force[k], 12);
  }
  put_bytes(out_, buf.data(), buf.size());
  if (!out_) throw std::runtime_error("failed to write trajectory output file " + path_ + ".");
}

void TrajectoryFile::flush() { out_.flush(); }

void write_final_state(const std::string& prefix, const char* units, uint64_t step,
                       const float lo[3], const float hi[3], const Engine::SlotView& sv,
                       const std::vector<int32_t>& type_by_tag) {
  if (prefix.empty()) throw InvalidArgument("output.final_state.prefix must not be empty.");
  const std::string path = prefix + ".state.beadsbin";
  std::ofstream out(path, std::ios::binary | std::ios::trunc);
  if (!out) throw std::runtime_error("failed to open final-state output file " + path + ".");
  const char magic[] = "BEADS_SNAPSHOT";
  put_bytes(out, magic, sizeof(magic) - 1);
  put<uint32_t>(out, kFormatVersion);
  put<uint32_t>(out, 4);  // real
  put<uint32_t>(out, 4);  // index
  put<uint32_t>(out, 4);  // image
  put<uint32_t>(out, 4);  // type
  put<uint32_t>(out, 4);  // tag
  put<uint32_t>(out, kEndianMarker);
  put_units(out, units);
  put<uint64_t>(out, step);
  const uint64_t n = sv.tag.size();
  put<uint64_t>(out, n);
  put_bytes(out, lo, 12);
  put_bytes(out, hi, 12);
  std::vector<float> f(n);
  std::vector<int32_t> iv(n);
  put_bytes(out, sv.tag.data(), 4 * n);
  for (uint64_t k = 0; k < n; ++k) iv[k] = type_by_tag[sv.tag[k] - 1];
  put_bytes(out, iv.data(), 4 * n);
  put_bytes(out, sv.mol.data(), 4 * n);
  for (uint64_t k = 0; k < n; ++k) f[k] = sv.vel[k].w;
  put_bytes(out, f.data(), 4 * n);
  const float4* arrays[2] = {sv.pos.data(), sv.vel.data()};
  for (const float4* a : arrays) {
    for (int c = 0; c < 3; ++c) {
      for (uint64_t k = 0; k < n; ++k) f[k] = c == 0 ? a[k].x : (c == 1 ? a[k].y : a[k].z);
      put_bytes(out, f.data(), 4 * n);
    }
  }
  for (int c = 0; c < 3; ++c) {
    for (uint64_t k = 0; k < n; ++k) iv[k] = c == 0 ? sv.img[k].x : (c == 1 ? sv.img[k].y : sv.img[k].z);
    put_bytes(out, iv.data(), 4 * n);
  }
  out.flush();
  if (!out) throw std::runtime_error("failed to write final-state output file " + path + ".");
}

std::string log_label(const std::string& label, const std::string& value) {
  // "  label<pad> : value" with the value starting at column 39.
  std::string line = "  " + label;
  const size_t target = 39 - 3;
  line += line.size() < target ? std::string(target - line.size(), ' ') : std::string(" ");
  return line + " : " + value;
}

LogSink::LogSink(int echo, const char* prefix) {
  screen_ = echo == BEADS_ECHO_SCREEN || echo == BEADS_ECHO_BOTH;
  file_ = echo == BEADS_ECHO_LOG || echo == BEADS_ECHO_BOTH;
  if (file_) {
    if (!prefix || !*prefix) throw InvalidArgument("output.log.prefix must be provided for file logging.");
    path_ = std::string(prefix) + ".log";
    out_.open(path_, std::ios::out | std::ios::trunc);
    if (!out_) throw std::runtime_error("failed to open log output file " + path_ + ".");
  }
}

void LogSink::message(const char* level, const std::string& text) {
  if (!active()) return;
  const bool gap = wrote_ && std::string(level) != "THERMO";
  const std::string line = std::string("[BEADS] ") + level + " " + text;
  if (screen_) {
    if (gap) std::cout << '\n';
    std::cout << line << '\n';
  }
  if (file_) {
    if (gap) out_ << '\n';
    out_ << line << '\n';
  }
  wrote_ = true;
}

void LogSink::thermo_row(const beads_observables& o, ThermoSchema schema) {
  if (!active()) return;
  auto col = [](const std::string& s) {
    std::ostringstream c;
    c << std::setw(16) << s;
    return c.str();
  };
  if (!header_) {
    std::string h = col("Step") + col("PotEng") + col("PairEng");
    if (schema.bond) h += col("BondEng");
    if (schema.angle) h += col("AngleEng");
    if (schema.dihedral) h += col("DihedEng");
    h += col("KinEng") + col("Temp") + col("Press");
    message("THERMO", h);
    header_ = true;
  }
  std::string r = col(std::to_string(o.step)) + col(real9(o.pe)) + col(real9(o.pair_pe));
  if (schema.bond) r += col(real9(o.bond_pe));
  if (schema.angle) r += col(real9(o.angle_pe));
  if (schema.dihedral) r += col(real9(o.dihedral_pe));
  r += col(real9(o.ke)) + col(real9(o.temp)) + col(real9(o.press));
  message("THERMO", r);
}

void LogSink::flush() {
  if (file_) out_.flush();
  if (screen_) std::cout.flush();
}

}  // namespace bb
