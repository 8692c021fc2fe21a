// Semtex binary field files (.fld / .rst / .chk / .frc): writeField /
// readField (src/misc.cpp:106-222) with the AuxField binary stream
// operators (src/auxfield.cpp:1021-1113).  Ten text header lines, each a
// 25-character value column and a label, then every field's nz planes of
// nel*np*np doubles in the writer's byte order.
#pragma once

#include <string>
#include <vector>

namespace stx {

struct FieldFile {
  std::string session;
  int np = 0, nz = 0, nel = 0, step = 0;
  double time = 0.0, dt = 0.0, kinvis = 0.0, beta = 0.0;
  std::string names;                       // one character per field
  std::vector<std::vector<double>> data;   // [field][nz*nel*np*np], physical space
};

// Append (or create) one dump.
void write_field(const std::string& path, const FieldFile& f, bool append = false);
// Read the first dump of a file (byte order from its header).
FieldFile read_field(const std::string& path);

}  // namespace stx
