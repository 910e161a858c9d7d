// Text trajectory loaders of the public C++ API (drop-in for the reference's
// include/txtReader.hpp:6-88).  Unlike the reference header the functions are inline, so
// the header can be included from several translation units.
#pragma once

#include <iostream>
#include <string>

#include "geometry_basics.hpp"
#include "rfd_txt_parse.hpp"

namespace rfd_txt {
inline Points load_points(const std::string& path, int cmp, int START, int LIMIT) {
  Points ret;
  ParseStats st = parse_file(
      path, cmp, START, LIMIT, [&](const std::vector<double>& c) { ret.push_back(Point(c)); },
      [&](const std::string& line) {
        std::cerr << "Warning: invalid double in line: " << line << std::endl;
      });
  if (!st.opened) std::cerr << "Failed to open file: " << path << std::endl;
  return ret;
}
}  // namespace rfd_txt

inline Points txtLoader2(const std::string& path, int START = 0, int LIMIT = 10000000) {
  return rfd_txt::load_points(path, 2, START, LIMIT);
}

inline Points txtLoader3(const std::string& path, int START = 0, int LIMIT = 10000000) {
  return rfd_txt::load_points(path, 3, START, LIMIT);
}
