// Geometry value types of the public C++ API (drop-in for the reference's
// include/geometry_basics.hpp:11-134): Point wraps a coordinate vector, Points is a
// vector of them, Interval is [begin, end] with begin > end meaning empty.
#pragma once

#include <cmath>
#include <cstddef>
#include <iostream>
#include <vector>

struct Point {
  std::vector<double> coordinates;

  inline Point() {}
  inline Point(const std::vector<double>& in) : coordinates{in} {}

  inline Point& operator-=(const Point& o) {
    for (std::size_t i = 0; i < coordinates.size(); ++i) coordinates[i] -= o.coordinates[i];
    return *this;
  }
  inline Point operator-(const Point& o) const {
    Point r = *this;
    r -= o;
    return r;
  }
  inline Point& operator+=(const Point& o) {
    for (std::size_t i = 0; i < coordinates.size(); ++i) coordinates[i] += o.coordinates[i];
    return *this;
  }
  inline Point operator+(const Point& o) const {
    Point r = *this;
    r += o;
    return r;
  }
  inline Point operator*(const double m) const {
    Point r;
    r.coordinates.resize(coordinates.size());
    for (std::size_t i = 0; i < coordinates.size(); ++i) r.coordinates[i] = coordinates[i] * m;
    return r;
  }
  inline Point& operator/=(double v) {
    for (auto& c : coordinates) c /= v;
    return *this;
  }
  // Squared Euclidean distance, summed in coordinate order.
  inline double dist_sqr(const Point& o) const {
    double s = 0.0;
    for (std::size_t i = 0; i < coordinates.size(); ++i) {
      const double t = coordinates[i] - o.coordinates[i];
      s += t * t;
    }
    return s;
  }
  inline double dist(const Point& o) const { return std::sqrt(dist_sqr(o)); }
  inline std::vector<double>& getCoordinates() { return coordinates; }
  inline const std::vector<double>& getCoordinates() const { return coordinates; }
  inline double operator[](std::size_t i) const { return coordinates[i]; }
  inline int size() const { return (int)coordinates.size(); }
};
typedef std::vector<Point> Points;
typedef std::vector<Points> multiPoints;

inline std::ostream& operator<<(std::ostream& out, const Point& p) {
  out << "(";
  for (std::size_t i = 0; i < p.coordinates.size(); ++i) out << (i ? ", " : "") << p.coordinates[i];
  return out << ")";
}

struct Interval {
  double begin;
  double end;
  Interval() : begin(1.), end(0.) {}
  Interval(double b, double e) : begin(b), end(e) {}
  inline bool operator<(const Interval& o) const {
    return begin < o.begin || (begin == o.begin && end < o.end);
  }
  inline bool is_empty() const { return begin > end; }
  inline bool intersects(const Interval& o) const {
    if (is_empty() || o.is_empty()) return false;
    return (o.begin >= begin && o.begin <= end) || (o.end >= begin && o.end <= end) ||
           (o.begin <= begin && o.end >= end);
  }
};
typedef std::vector<Interval> Intervals;

inline std::ostream& operator<<(std::ostream& out, const Interval& iv) {
  return out << "[" << iv.begin << ", " << iv.end << "]";
}
