#include "session.hpp"

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace stx {

namespace {

std::string upper(std::string s) {
  for (auto& c : s) c = static_cast<char>(std::toupper(static_cast<unsigned char>(c)));
  return s;
}

std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

// Body of section <NAME ...> ... </NAME>; returns false if absent.
bool section(const std::string& text, const std::string& name, std::string& body) {
  const std::string U = upper(text);
  const std::string open = "<" + name;
  size_t p = 0;
  while ((p = U.find(open, p)) != std::string::npos) {
    size_t q = p + open.size();
    if (q < U.size() && (U[q] == '>' || std::isspace(static_cast<unsigned char>(U[q])))) break;
    p = q;
  }
  if (p == std::string::npos) return false;
  size_t gt = U.find('>', p);
  size_t end = U.find("</" + name, gt);
  if (gt == std::string::npos || end == std::string::npos)
    throw std::runtime_error("FEML: unterminated section " + name);
  body = text.substr(gt + 1, end - gt - 1);
  return true;
}

// Integer attribute `attr=` of the opening tag of section NAME
// (FEML::attribute, src/feml.cpp:258-300); -1 when the tag lacks it.
int attribute(const std::string& text, const std::string& name, const std::string& attr) {
  const std::string U = upper(text);
  const std::string open = "<" + name;
  size_t p = 0;
  while ((p = U.find(open, p)) != std::string::npos) {
    size_t q = p + open.size();
    if (q < U.size() && (U[q] == '>' || std::isspace(static_cast<unsigned char>(U[q])))) break;
    p = q;
  }
  if (p == std::string::npos) return -1;
  const size_t gt = U.find('>', p);
  const std::string tag = U.substr(p, gt == std::string::npos ? std::string::npos : gt - p);
  const size_t a = tag.find(upper(attr) + "=");
  if (a == std::string::npos) return -1;
  return std::atoi(tag.c_str() + a + attr.size() + 1);
}

std::vector<std::string> lines(const std::string& body) {
  std::vector<std::string> out;
  std::istringstream is(body);
  std::string ln;
  while (std::getline(is, ln)) {
    std::string t = trim(ln);
    if (!t.empty() && t[0] != '#') out.push_back(t);
  }
  return out;
}

// Content between <X> and </X> on one line; returns tag letter.
char tagged(const std::string& ln, std::string& inner, std::string& before) {
  size_t a = ln.find('<');
  size_t b = ln.find('>', a);
  size_t c = ln.find("</", b);
  if (a == std::string::npos || b == std::string::npos || c == std::string::npos)
    throw std::runtime_error("FEML: malformed tagged line: " + ln);
  before = trim(ln.substr(0, a));
  inner = trim(ln.substr(b + 1, c - b - 1));
  return trim(ln.substr(a + 1, b - a - 1))[0];
}

}  // namespace

std::string Session::user_value(const std::string& key) const {
  const std::string K = upper(key);
  for (const auto& ln : user) {
    std::istringstream is(ln);
    std::string first;
    is >> first;
    if (upper(first) == K) {
      std::string rest;
      std::getline(is, rest);
      rest = trim(rest);
      if (!rest.empty() && rest[0] == '=') rest = trim(rest.substr(1));
      return rest;
    }
    size_t eq = ln.find('=');
    if (eq != std::string::npos && upper(trim(ln.substr(0, eq))) == K)
      return trim(ln.substr(eq + 1));
  }
  return "";
}

Session read_session(const std::string& path, const std::string& overrides) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("couldn't open session file " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string text = ss.str();
  Session S;
  S.path = path;
  size_t slash = path.find_last_of('/');
  S.name = slash == std::string::npos ? path : path.substr(slash + 1);

  std::string body;
  if (section(text, "TOKENS", body)) {
    for (const auto& ln : lines(body))
      if (ln.find('=') != std::string::npos) S.tokens.assign(ln);
  }
  if (!overrides.empty()) {
    std::istringstream is(overrides);
    std::string a;
    while (std::getline(is, a, ';'))
      if (trim(a).size()) S.tokens.assign(a);
  }
  // src/feml.cpp:310-318
  if (S.tokens.ivalue("IO_FLD") > S.tokens.ivalue("N_STEP"))
    S.tokens.set("IO_FLD", S.tokens.value("N_STEP"));
  if (S.tokens.ivalue("N_TIME") > 3) S.tokens.set("N_TIME", 3);

  if (!section(text, "FIELDS", body)) throw std::runtime_error("FEML: no FIELDS section");
  for (char c : body)
    if (std::isalpha(static_cast<unsigned char>(c))) S.fields.push_back(c);

  if (section(text, "GROUPS", body)) {
    for (const auto& ln : lines(body)) {
      std::istringstream is(ln);
      int id;
      std::string g, d;
      is >> id >> g >> d;
      S.groups[g[0]] = d;
    }
  }
  // HISTORY (Analyser::Analyser, src/analysis.cpp:108-134): NUMBER
  // points read as "id x y z" from the section's start
  if (section(text, "HISTORY", body)) {
    const int n = attribute(text, "HISTORY", "NUMBER");
    if (n < 0) throw std::runtime_error("FEML: HISTORY needs NUMBER=");
    std::istringstream is(body);
    for (int i = 0; i < n; ++i) {
      HistoryPoint h;
      if (!(is >> h.id >> h.x >> h.y >> h.z)) throw std::runtime_error("FEML: short HISTORY section");
      S.history.push_back(h);
    }
  }
  if (section(text, "BCS", body)) {
    auto L = lines(body);
    for (size_t i = 0; i < L.size();) {
      std::istringstream is(L[i]);
      int id, nf;
      std::string g;
      is >> id >> g >> nf;
      for (int j = 0; j < nf; ++j) {
        std::string inner, before;
        char kind = tagged(L[i + 1 + j], inner, before);
        BCSpec bc;
        bc.kind = kind;
        char fld = inner[0];
        size_t eq = inner.find('=');
        bc.expr = eq == std::string::npos ? "" : trim(inner.substr(eq + 1));
        S.bcs[g[0]][fld] = bc;
      }
      i += 1 + nf;
    }
  }
  if (!section(text, "NODES", body)) throw std::runtime_error("FEML: no NODES section");
  {
    auto L = lines(body);
    S.nodes.resize(L.size());
    for (const auto& ln : L) {
      std::istringstream is(ln);
      int id;
      double x, y, z;
      is >> id >> x >> y >> z;
      if (id < 1 || id > static_cast<int>(L.size()))
        throw std::runtime_error("FEML: node id out of range");
      S.nodes[id - 1] = {x, y, z};
    }
  }
  if (!section(text, "ELEMENTS", body)) throw std::runtime_error("FEML: no ELEMENTS section");
  {
    auto L = lines(body);
    S.elements.resize(L.size());
    for (const auto& ln : L) {
      std::string inner, before;
      char kind = tagged(ln, inner, before);
      if (kind != 'Q') throw std::runtime_error("unrecognized element tag");
      int id = std::stoi(before);
      std::istringstream is(inner);
      std::array<int, 4> v{};
      for (auto& n : v) {
        is >> n;
        if (n < 1 || n > static_cast<int>(S.nodes.size()))
          throw std::runtime_error("FEML: element node out of range");
        --n;
      }
      if (id < 1 || id > static_cast<int>(L.size()))
        throw std::runtime_error("FEML: element id out of range");
      S.elements[id - 1] = v;
    }
  }
  if (section(text, "SURFACES", body)) {
    for (const auto& ln : lines(body)) {
      std::string inner, before;
      char kind = tagged(ln, inner, before);
      std::istringstream is(before);
      int id, e, s;
      is >> id >> e >> s;
      Surface sf;
      sf.elmt = e - 1;
      sf.side = s - 1;
      sf.kind = kind;
      if (kind == 'B') {
        sf.group = inner[0];
      } else if (kind == 'P') {
        std::istringstream js(inner);
        js >> sf.mate_elmt >> sf.mate_side;
        --sf.mate_elmt;
        --sf.mate_side;
      } else {
        throw std::runtime_error("couldn't recognize Surface tag");
      }
      S.surfaces.push_back(sf);
    }
  }
  if (section(text, "CURVES", body)) S.has_curves = !lines(body).empty();
  if (section(text, "USER", body)) S.user = lines(body);
  if (section(text, "FORCE", body)) {
    S.has_force = true;
    std::istringstream is(body);
    std::string ln;
    std::getline(is, ln);  // the rest of the opening tag's line
    while (std::getline(is, ln)) {
      if (!ln.empty() && ln.back() == '\r') ln.pop_back();
      S.force.push_back(ln);
    }
  }
  return S;
}

bool Session::force_value(const std::string& token, std::string& value) const {
  for (size_t k = 0; k < force.size(); ++k) {
    const std::string& s = force[k];
    if (!s.empty() && s[0] == '#') {
      ++k;  // the reference reads past the comment line and the one after it
      continue;
    }
    auto delim = [](char c) { return c == '\t' || c == '=' || c == ' '; };
    size_t a = 0;
    while (a < s.size() && delim(s[a])) ++a;
    if (a == s.size()) continue;
    size_t b = a;
    while (b < s.size() && !delim(s[b])) ++b;
    if (s.compare(a, b - a, token) != 0 || b - a != token.size()) continue;
    size_t c = b < s.size() ? b + 1 : b;  // the delimiter that ended the word
    while (c < s.size() && s[c] == '=') ++c;
    size_t d = c;
    while (d < s.size() && s[d] != '=') ++d;
    if (c == d) return false;
    value = s.substr(c, d - c);
    return true;
  }
  return false;
}

}  // namespace stx
