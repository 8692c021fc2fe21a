#include "fieldfile.hpp"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace stx {

namespace {

bool host_little() {
  const uint16_t one = 1;
  unsigned char b;
  std::memcpy(&b, &one, 1);
  return b == 1;
}

std::string column(const std::string& v, const char* label) {
  char buf[128];
  std::snprintf(buf, sizeof(buf), "%-25s %s\n", v.c_str(), label);
  return buf;
}

std::string gfmt(double v) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%.6g", v);
  return buf;
}

}  // namespace

void write_field(const std::string& path, const FieldFile& f, bool append) {
  const size_t n = static_cast<size_t>(f.np) * f.np * f.nz * f.nel;
  if (f.data.size() != f.names.size()) throw std::runtime_error("write_field: names and data differ");
  for (const auto& d : f.data)
    if (d.size() != n) throw std::runtime_error("write_field: field size does not match the header");
  std::ofstream out(path, append ? std::ios::binary | std::ios::app : std::ios::binary | std::ios::trunc);
  if (!out) throw std::runtime_error("can't open field file " + path);
  char created[64];
  const std::time_t now = std::time(nullptr);
  std::strftime(created, sizeof(created), "%a %b %d %H:%M:%S %Y", std::localtime(&now));
  std::ostringstream hdr;
  hdr << column(f.session, "Session") << column(created, "Created")
      << column(std::to_string(f.np) + " " + std::to_string(f.np) + " " + std::to_string(f.nz) + " " +
                    std::to_string(f.nel),
                "Nr, Ns, Nz, Elements")
      << column(std::to_string(f.step), "Step") << column(gfmt(f.time), "Time")
      << column(gfmt(f.dt), "Time step") << column(gfmt(f.kinvis), "Kinvis") << column(gfmt(f.beta), "Beta")
      << column(f.names, "Fields written")
      << column(host_little() ? "binary IEEE little-endian" : "binary IEEE big-endian", "Format");
  const std::string h = hdr.str();
  out.write(h.data(), static_cast<std::streamsize>(h.size()));
  for (const auto& d : f.data) out.write(reinterpret_cast<const char*>(d.data()), sizeof(double) * n);
  if (!out) throw std::runtime_error("write failed: " + path);
}

FieldFile read_field(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw std::runtime_error("can't open field file " + path);
  std::string line[10];
  for (auto& l : line)
    if (!std::getline(in, l)) throw std::runtime_error(path + ": short header");
  FieldFile f;
  std::istringstream(line[0]) >> f.session;
  int ns = 0;
  std::istringstream(line[2]) >> f.np >> ns >> f.nz >> f.nel;
  std::istringstream(line[3]) >> f.step;
  std::istringstream(line[4]) >> f.time;
  std::istringstream(line[5]) >> f.dt;
  std::istringstream(line[6]) >> f.kinvis;
  std::istringstream(line[7]) >> f.beta;
  std::istringstream(line[8]) >> f.names;
  const bool swap = (line[9].find("big") != std::string::npos) == host_little();
  const size_t n = static_cast<size_t>(f.np) * f.np * f.nz * f.nel;
  for (size_t k = 0; k < f.names.size(); ++k) {
    std::vector<double> d(n);
    in.read(reinterpret_cast<char*>(d.data()), static_cast<std::streamsize>(sizeof(double) * n));
    if (!in) throw std::runtime_error(path + ": truncated field");
    if (swap)
      for (auto& v : d) {
        unsigned char* b = reinterpret_cast<unsigned char*>(&v);
        for (int i = 0; i < 4; ++i) std::swap(b[i], b[7 - i]);
      }
    f.data.push_back(std::move(d));
  }
  return f;
}

}  // namespace stx
