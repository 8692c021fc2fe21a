// FEML session-file reader.
//
// Reads the sections the reference reads for the dns / elliptic hot path
// (src/feml.cpp:64-330, src/mesh.cpp:129-470, src/bcmgr.cpp:100-110):
// TOKENS, FIELDS, GROUPS, HISTORY, BCS, NODES, ELEMENTS (<Q> quads), SURFACES
// (<B> boundary group or <P> periodic mate), USER, FORCE (dns/fieldforce.cpp:
// 31-73).  CURVES are recorded as present and rejected by the mesh builder
// (straight sides only).
#pragma once

#include <array>
#include <map>
#include <string>
#include <vector>

#include "expr.hpp"

namespace stx {

struct BCSpec {
  char kind = 0;        // 'D' essential, 'N' natural, 'H' high-order pressure ...
  std::string expr;     // value or function of x, y, z, t
};

struct Surface {
  int elmt = 0, side = 0;  // zero-based element and side
  char kind = 0;           // 'B' boundary group, 'P' periodic
  char group = 0;          // for 'B'
  int mate_elmt = -1, mate_side = -1;  // for 'P'
};

// A history point of the HISTORY section (Analyser::Analyser,
// src/analysis.cpp:108-134): tag and location.
struct HistoryPoint {
  int id = 0;
  double x = 0.0, y = 0.0, z = 0.0;
};

struct Session {
  std::string path, name;
  TokenTable tokens;
  std::string fields;                                // e.g. "uvwp" or "c"
  std::map<char, std::string> groups;                // group -> descriptor
  std::map<char, std::map<char, BCSpec>> bcs;        // group -> field -> BC
  std::vector<std::array<double, 3>> nodes;
  std::vector<std::array<int, 4>> elements;          // zero-based node ids
  std::vector<Surface> surfaces;
  std::vector<std::string> user;                     // USER section lines
  bool has_curves = false;
  bool has_force = false;                            // <FORCE> section present
  std::vector<std::string> force;                    // its raw lines
  std::vector<HistoryPoint> history;                 // HISTORY section, in order

  // FEML::valueFromSection (src/feml.cpp:430-560) on the FORCE section: the
  // text after `token` on the first line whose first word is `token` (words
  // end at tab, '=' or space; the value is what follows up to the next '=').
  // A line starting with '#' is skipped together with the line after it, as
  // the reference skips them.  False if absent.
  bool force_value(const std::string& token, std::string& value) const;

  // USER line "key value" (elliptic forcing/exact) or "name = expr".
  std::string user_value(const std::string& key) const;
};

// `overrides` holds "NAME=expr" assignments separated by ';' applied after
// the <TOKENS> section (the role of command-line token overrides).
Session read_session(const std::string& path, const std::string& overrides = "");

}  // namespace stx
