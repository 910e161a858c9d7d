// Curve type of the public C++ API (drop-in for the reference's include/curve.hpp:9-49 and
// src/curve.cpp:3-18): an ordered list of points of a fixed dimension.
#pragma once

#include <cstdio>
#include <iostream>

#include "geometry_basics.hpp"

class Curve {
 public:
  typedef unsigned long index_type;

  Curve(unsigned int dimensions) : number_dimensions{dimensions} {}
  Curve(const Points& pts, unsigned int dimensions) : points(pts), number_dimensions(dimensions) {
    if (points.empty()) std::cerr << "warning: constructed empty curve" << std::endl;
  }

  inline std::size_t size() const { return points.size(); }
  inline bool empty() const { return points.empty(); }
  inline std::size_t dimensions() const { return number_dimensions; }
  inline Point const& operator[](const std::size_t i) const { return points[i]; }
  inline Point front() const { return points.front(); }
  inline Point back() const { return points.back(); }
  inline void push_back(const Point& p) { points.push_back(p); }
  // Translates every point by -p (the reference also prints debugging lines here).
  inline void recenter(const Point& p) {
    for (auto& q : points) q -= p;
  }
  inline Points::iterator begin() { return points.begin(); }
  inline Points::iterator end() { return points.end(); }
  inline Points::const_iterator begin() const { return points.cbegin(); }
  inline Points::const_iterator end() const { return points.cend(); }

 private:
  Points points;
  unsigned int number_dimensions;
};

class Curves : public std::vector<Curve> {
 public:
  inline Curve get(std::size_t i) const { return this->operator[](i); }
};

inline std::ostream& operator<<(std::ostream& out, const Curve& c) {
  out << "[";
  for (std::size_t i = 0; i < c.size(); ++i) out << (i ? ", " : "") << c[i];
  return out << "]";
}
