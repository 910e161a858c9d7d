// Text trajectory parser shared by txtLoader2/3 (include/txtReader.hpp) and rfd_load_txt.
//
// Format and rules of the reference loader (include/txtReader.hpp:6-88 of the reference):
// one point per line, coordinates separated by ',', each parsed with std::stod (a token
// that does not parse is reported and skipped); a line with no coordinate is ignored; the
// point counter advances for every non-empty point, parsing stops once LIMIT points were
// counted, points whose counter is below START are skipped; a point equal to the last kept
// point in its first `cmp` coordinates (2 for txtLoader2, 3 for txtLoader3) is dropped.
#pragma once

#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace rfd_txt {

struct ParseStats {
  bool opened = false;
  long long bad_tokens = 0;
};

// on_point(const std::vector<double>& coords) is called for every kept point;
// on_bad(const std::string& line) for every token std::stod rejects.
template <class OnPoint, class OnBad>
inline ParseStats parse_file(const std::string& path, int cmp, int START, int LIMIT,
                             OnPoint on_point, OnBad on_bad) {
  ParseStats st;
  std::ifstream fin(path);
  if (!fin.is_open()) return st;
  st.opened = true;
  std::string line;
  int count = 0;
  bool have_last = false;
  std::vector<double> last;
  while (std::getline(fin, line)) {
    if (count >= LIMIT) break;
    std::stringstream ss(line);
    std::string token;
    std::vector<double> pt;
    while (std::getline(ss, token, ',')) {
      try {
        pt.push_back(std::stod(token));
      } catch (const std::exception&) {
        ++st.bad_tokens;
        on_bad(line);
      }
    }
    if (pt.empty()) continue;
    ++count;
    if (count < START) continue;
    bool keep = !have_last;
    if (have_last) {
      for (int k = 0; k < cmp; ++k) {
        const double a = k < (int)last.size() ? last[k] : 0.0;
        const double b = k < (int)pt.size() ? pt[k] : 0.0;
        if (a != b) keep = true;
      }
    }
    if (keep) {
      last = pt;
      have_last = true;
      on_point(pt);
    }
  }
  return st;
}

}  // namespace rfd_txt
