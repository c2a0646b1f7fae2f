// File-based set-up and VTK output: FlowLB's path from Geometry.txt and
// OptionsCalc.txt to the solver's inputs (geometry flags, tau, body force,
// inlet velocity, loop bounds), and its ASCII VTK ImageData writer.
//
// Reference behaviour followed here (FlowLB, src/):
//   io/reader.cpp:25-139     option-line splitting and substring rules
//   io/reader.cpp:261-556    OptionsCalc.txt options and their checks
//   io/reader.cpp:558-658    INITIAL_CONDITION_FLAG(n).* shapes
//   io/reader.cpp:766-1217   Geometry.txt: POINT, SIZE, CDW, OBSTACLE
//   geometry/mesh.cpp:44-51  lattice size from the bounding box
//   geometry/shapes.cpp      rectangle (rotated), circle, CSV polygon, CDW tests
//   initData.h:42-66,220-317 the geometry sweep that writes the cell flags
//   initData.cpp:13-124      the free-surface flag sweep (interface layer)
//   utils.cpp:7-82           SI <-> lattice unit conversion
//   cuda/cudaInitData.cu:57-82  tau and the body force as float constants
//   cuda/runCuda.cu:460-528  headless loops: T+1 steps, save every tSave
//   io/writer.cpp:15-252     VTIWriter: file layout, number formatting, series
//
// Everything here is host code.  Parse errors are reported with the
// reference's own messages in flb_setup::error; where the reference reads out
// of bounds or crashes on malformed input (an END_POSITION_SHAPES equal to the
// point count, an unparsable number outside a try block, a CSV row with one
// column) this code reports an error instead.

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/flowlb.h"

namespace {

// Cell flags (src/utils.h:91-108).
constexpr uint8_t kFluid = 0x01, kGas = 0x02, kInterface = 0x04, kWall = 0x08, kInlet = 0x20, kOutlet = 0x40;
constexpr uint8_t kNone = 100;
constexpr double kPi = 3.141592653589793;
constexpr double kEps = 1e-12;       // Shape::m_Epsilon, CDW::m_Epsilon, initData's epsilon
constexpr uint32_t kMaxThreadsPerBlock = 1024;  // B200

struct SetupError {
  flb_status status;
  std::string msg;
};

[[noreturn]] void fail(const std::string& m, flb_status s = FLB_ERR_INVALID_ARGUMENT) { throw SetupError{s, m}; }

std::string fmt_line(const char* prefix, const char* text, unsigned line) {
  char buf[320];
  std::snprintf(buf, sizeof buf, text, line);
  return std::string(prefix) + " " + buf;
}

// ---- number parsing with the semantics of std::stod / stof / stoi --------
// (leading whitespace and sign accepted, longest valid prefix, error when no
// digits were read or the value is out of range) and of std::from_chars with
// chars_format::general (no leading whitespace, no '+', no hexadecimal).

bool parse_double(const std::string& s, double& v) {
  const char* b = s.c_str();
  char* e = nullptr;
  errno = 0;
  v = std::strtod(b, &e);
  return e != b && errno != ERANGE;
}

bool parse_float(const std::string& s, float& v) {
  const char* b = s.c_str();
  char* e = nullptr;
  errno = 0;
  v = std::strtof(b, &e);
  return e != b && errno != ERANGE;
}

bool parse_int(const std::string& s, int& v) {
  const char* b = s.c_str();
  char* e = nullptr;
  errno = 0;
  const long r = std::strtol(b, &e, 10);
  if (e == b || errno == ERANGE || r < -2147483648L || r > 2147483647L) return false;
  v = (int)r;
  return true;
}

bool parse_chars_general(const std::string& s, double& v) {
  if (s.empty() || s[0] == '+' || std::isspace((unsigned char)s[0])) return false;
  const size_t k = (s[0] == '-') ? 1 : 0;
  if (s.size() > k + 1 && s[k] == '0' && (s[k + 1] == 'x' || s[k + 1] == 'X')) {
    v = k ? -0.0 : 0.0;  // general format reads the leading "0" only
    return true;
  }
  if (k < s.size() && std::isspace((unsigned char)s[k])) return false;
  return parse_double(s, v);
}

// ---- substring rules of Reader::extractString (reader.cpp:67-139) --------

long find_or_minus1(const std::string& s, char c, size_t from = 0) {
  const size_t p = s.find(c, from);
  return p == std::string::npos ? -1L : (long)p;
}

// Text before the first `d`; the whole string when `d` is absent.
std::string before(const std::string& s, char d) {
  const long p = find_or_minus1(s, d);
  return p < 0 ? s : s.substr(0, (size_t)p);
}

// Text from two characters after the first `d` (the attribute after ").").
std::string attribute_after(const std::string& s, char d, unsigned line) {
  const long p = find_or_minus1(s, d);
  const size_t start = (size_t)(p + 2);
  if (start > s.size())
    fail("The option in the geometry's file in the line " + std::to_string(line) + " is incorrect");
  return s.substr(start);
}

// Text between the first `a` and the first `b`; to the end when `b` comes
// first or is absent, from the start when `a` is absent.
std::string between(const std::string& s, char a, char b) {
  const long ia = find_or_minus1(s, a), ib = find_or_minus1(s, b);
  const size_t start = (size_t)(ia + 1);
  const long n = ib - ia - 1;
  return n < 0 ? s.substr(start) : s.substr(start, (size_t)n);
}

// "(x,y,z)": x between '(' and the first ',', y between the first two commas,
// z after the second comma to the end.  False when a comma is missing.
bool split_triple(const std::string& v, std::string& x, std::string& y, std::string& z) {
  const long c1 = find_or_minus1(v, ',');
  if (c1 < 0) return false;
  const long c2 = find_or_minus1(v, ',', (size_t)c1 + 1);
  if (c2 < 0) return false;
  x = between(v, '(', ',');
  y = v.substr((size_t)c1 + 1, (size_t)(c2 - c1 - 1));
  z = v.substr((size_t)c2 + 1);
  return true;
}

std::string strip_space(const std::string& s) {
  std::string o;
  o.reserve(s.size());
  for (char c : s)
    if (!std::isspace((unsigned char)c)) o.push_back(c);
  return o;
}

// Reader::splitString (reader.cpp:25-58): drop the comment after '#', split at
// '=' (at most two parts), remove all whitespace from each part.
bool split_option(const std::string& raw, std::string& key, std::string& value) {
  std::string s = raw;
  const size_t hash = s.find('#');
  if (hash != std::string::npos) s = s.substr(0, hash);
  key.clear();
  value.clear();
  std::vector<std::string> parts;
  size_t start = 0;
  while (start < s.size()) {
    const size_t p = s.find('=', start);
    if (p == std::string::npos) {
      parts.push_back(s.substr(start));
      break;
    }
    parts.push_back(s.substr(start, p - start));
    start = p + 1;
  }
  if (parts.size() > 2) return false;
  if (parts.size() > 0) key = strip_space(parts[0]);
  if (parts.size() > 1) value = strip_space(parts[1]);
  return true;
}

// ---- shapes (geometry/shapes.cpp) ----------------------------------------

enum class ShapeKind { Circle, Rectangle, Polygon };

struct Shape {
  ShapeKind kind;
  double x0 = 0, y0 = 0, z0 = 0;
  double xrot = 0, yrot = 0, zrot = 0;
  // circle
  double radius = 0, thickness = 0;
  // rectangle
  double height = 0, xwidth = 0, zwidth = 0;
  double bxmin = 0, bxmax = 0, bymin = 0, bymax = 0, bzmin = 0, bzmax = 0;
  double rx[2] = {0, 0}, ry[2] = {0, 0};
  bool rotate = false;
  // polygon (CSV_2D)
  std::string filename;
  std::vector<double> px, py;
  double area = 0, cx = 0, cy = 0;

  explicit Shape(ShapeKind k) : kind(k) {}

  // Shape::setValue of the three classes: each ignores what it does not hold.
  void set_position(double x, double y, double z) {
    x0 = x;
    y0 = y;
    if (kind != ShapeKind::Polygon) z0 = z;
  }
  void set_rotation(double x, double y, double z) {
    if (kind == ShapeKind::Rectangle) {
      xrot = x;
      yrot = y;
      zrot = z;
    } else if (kind == ShapeKind::Polygon) {
      zrot = z;
    }
  }

  // RectangleShape::initShape (shapes.cpp:58-116), 2D.
  void init_rectangle() {
    rotate = !(std::abs(zrot - 0.0) <= 1e-6);
    rx[0] = std::cos(-zrot);
    rx[1] = std::sin(-zrot);
    ry[0] = std::sin(-zrot);
    ry[1] = std::cos(-zrot);
    bxmax = x0 + xwidth / 2.0 + kEps;
    bxmin = x0 - xwidth / 2.0 - kEps;
    bymax = y0 + height / 2.0 + kEps;
    bymin = y0 - height / 2.0 - kEps;
    bzmax = z0 + zwidth / 2.0 + kEps;
    bzmin = z0 - zwidth / 2.0 - kEps;
  }

  // Imported2DShape::initShape (shapes.cpp:154-195): reads "x;y" rows from
  // <directory>/<name>.csv, moves the polygon's centroid to (x0, y0) and
  // rotates it by zrot about the centroid.
  void init_polygon(const std::filesystem::path& dir) {
    const std::string path = dir.string() + "/" + filename;
    std::ifstream in(path);
    if (!in.is_open()) fail("Error opening the file: " + path, FLB_ERR_IO);
    std::vector<std::string> lines;
    std::string l;
    while (std::getline(in, l))
      if (!l.empty()) lines.push_back(l);
    if (lines.empty()) fail("Error, the file " + path + " is empty", FLB_ERR_IO);
    if (lines.size() < 3) fail("Error, the file " + path + " doesn't have the minimun nmuber of lines with data");
    unsigned row_no = 1;
    for (std::string row : lines) {
      row.erase(std::remove(row.begin(), row.end(), ' '), row.end());
      const size_t sc = row.find(';');
      const std::string xs = row.substr(0, sc);
      if (sc == std::string::npos) fail("Error converting the y coordinate in the line " + std::to_string(row_no) +
                                        " of the file: " + path);
      const size_t sc2 = row.find(';', sc + 1);
      const std::string ys = row.substr(sc + 1, sc2 == std::string::npos ? std::string::npos : sc2 - sc - 1);
      double x = 0, y = 0;
      if (!parse_chars_general(xs, x))
        fail("Error converting the x coordinate in the line " + std::to_string(row_no) + " of the file: " + path);
      if (!parse_chars_general(ys, y))
        fail("Error converting the y coordinate in the line " + std::to_string(row_no) + " of the file: " + path);
      px.push_back(x);
      py.push_back(y);
      row_no++;
    }
    // area and centroid (shoelace), both taken as absolute values
    const size_t n = px.size();
    for (size_t i = 0; i + 1 < n; i++) {
      const double p = px[i] * py[i + 1] - px[i + 1] * py[i];
      area += p;
      cx += (px[i] + px[i + 1]) * p;
      cy += (py[i] + py[i + 1]) * p;
    }
    {
      const double p = (px[n - 1] * py[0] - px[0] * py[n - 1]);
      area += p;
      cx += (px[n - 1] + px[0]) * p;
      cy += (py[n - 1] + py[0]) * p;
    }
    area *= 0.5;
    area = area < 0 ? -area : area;
    cx /= (6.0 * area);
    cx = cx < 0 ? -cx : cx;
    cy /= (6.0 * area);
    cy = cy < 0 ? -cy : cy;
    // move and rotate; the bounding box starts at (0, 0) and each vertex
    // updates its maximum, or else its minimum (shapes.cpp:262-295)
    const bool rot = !(std::abs(zrot - 0.0) <= 1e-6);
    const double c = std::cos(zrot), s = std::sin(zrot);
    for (size_t i = 0; i < n; i++) {
      double& x = px[i];
      double& y = py[i];
      x -= cx;
      y -= cy;
      if (rot) {
        const double prev = x;
        x = x * c - y * s;
        y = prev * s + y * c;
      }
      x += x0;
      y += y0;
      if (x > bxmax) bxmax = x;
      else if (x < bxmin) bxmin = x;
      if (y > bymax) bymax = y;
      else if (y < bymin) bymin = y;
    }
    bxmax += kEps;
    bxmin -= kEps;
    bymax += kEps;
    bymin -= kEps;
  }

  bool inside(double x, double y, double z) const {
    switch (kind) {
      case ShapeKind::Circle: {  // shapes.cpp:26-40, 2D branch
        const double d2 = (y - y0) * (y - y0) + (x - x0) * (x - x0);
        return !(d2 > (radius * radius + kEps));
      }
      case ShapeKind::Rectangle: {  // shapes.cpp:118-137
        if (rotate) {
          const double prevX = (x - x0), prevY = (y - y0);
          x = prevX * rx[0] - prevY * rx[1];
          y = prevX * ry[0] + prevY * ry[1];
          x += x0;
          y += y0;
        }
        return !(x > bxmax || x < bxmin || y > bymax || y < bymin || z > bzmax || z < bzmin);
      }
      case ShapeKind::Polygon: {  // shapes.cpp:197-212: box, then crossing number
        if (x > bxmax || x < bxmin || y > bymax || y < bymin) return false;
        bool in = false;
        const size_t n = px.size();
        for (size_t i = 0, j = n - 1; i < n; j = i++) {
          if (((py[i] > y) != (py[j] > y)) && (x < (px[j] - px[i]) * (y - py[i]) / (py[j] - py[i]) + px[i])) in = !in;
        }
        return in;
      }
    }
    return false;
  }
};

struct Point {
  double x, y, z;
};

enum class CdwKind { Circle, Rectangle };

struct Cdw {
  CdwKind kind;
  double radius = 0, height = 0, width = 0;

  // CircularCDW / RectangularCDW::isNodeInside (shapes.cpp:405-449), 2D.
  bool inside(double x, double y, double z, const std::vector<Point>& p, uint32_t b) const {
    if (kind == CdwKind::Circle) {
      // squared distance from the node to the base line raised by the radius
      const double qx = x - p[b].x, qy = y - (p[b].y + radius), qz = z - p[b].z;
      const double vx = p[b - 1].x - p[b].x, vy = p[b - 1].y - p[b].y, vz = p[b - 1].z - p[b].z;
      const double cx = qy * vz - qz * vy, cy = qz * vx - qx * vz, cz = qx * vy - qy * vx;
      const double d2 = (cx * cx + cy * cy + cz * cz) / (vx * vx + vy * vy + vz * vz);
      return d2 <= (radius * radius + kEps);
    }
    const double slope = (p[b].y - p[b - 1].y) / (p[b].x - p[b - 1].x);
    const double ydown = p[b - 1].y + (x - p[b - 1].x) * slope;
    return y >= (ydown - kEps) && y <= (ydown + kEps);
  }
};

// ---- the mesh and the options --------------------------------------------

struct Mesh {
  std::vector<Point> points;
  std::vector<Cdw> cdws;
  std::vector<Shape> obstacles, initial;
  double size = 0;
  bool size_set = false;
  bool is3d = false;
  long idx_init = -1, idx_end = -1;
  double xmax = 0, xmin = 0, ymax = 0, ymin = 0, zmax = 0, zmin = 0;
  uint32_t nx = 0, ny = 0, nz = 1;
};

struct Options {
  int type_analysis = 0;
  int graphics = 0;  // 0 NONE, 1 OPENGL
  bool free_surface = false;
  int collision = 0;
  bool surface_tension = false;
  int precision = 32;
  double ref_velocity_lb = 0.1, ref_velocity_si = 1.0;
  bool use_force = false, subgrid = false;
  double acc[3] = {0, 0, 0}, vforce[3] = {0, 0, 0};
  double flow = 0, relaxation_time = 0;
  double vel_si[3] = {0, 0, 0};
  double nu = 0, density = 0;
  float time_simulation = 0, time_save = 0;
  uint32_t block[3] = {0, 0, 0};
  uint8_t left = kNone, right = kNone, up = kNone, down = kNone;
};

constexpr const char* kGeoErr = "[GEOMETRY OPTIONS ERROR]";
constexpr const char* kCalcErr = "[CALCULATION OPTIONS ERROR]";

int element_number(const std::string& key, unsigned line) {
  int n = 0;
  if (!parse_int(between(key, '(', ')'), n) || n < 1)
    fail("The option in the geometry's file in the line " + std::to_string(line) + " is incorrect");
  return n;
}

double num(const std::string& s, const char* prefix, unsigned line) {
  double v = 0;
  if (!parse_double(s, v)) fail(fmt_line(prefix, "The value in the line %d is invalid", line));
  return v;
}

void triple(const std::string& v, double out[3], const char* prefix, const char* what, unsigned line) {
  std::string a, b, c;
  if (!split_triple(v, a, b, c) || !parse_double(a, out[0]) || !parse_double(b, out[1]) || !parse_double(c, out[2]))
    fail(std::string(prefix) + " The value of the " + what + " in the line " + std::to_string(line) + " is invalid");
}

// GeometryReader::getMeshElements (reader.cpp:783-830)
void geo_mesh_elements(Mesh& m, const std::string& key, const std::string& value, unsigned line) {
  const std::string type = before(key, '(');
  if (type == "POINT") {
    const int n = element_number(key, line);
    if ((int)m.points.size() >= n)
      fail(fmt_line(kGeoErr, "The numeration of the point in the line %d is not correct, maybe it is repeated", line));
    double c[3];
    triple(value, c, kGeoErr, "point", line);
    if (c[0] > m.xmax) m.xmax = c[0];
    if (c[0] < m.xmin) m.xmin = c[0];
    if (c[1] > m.ymax) m.ymax = c[1];
    if (c[1] < m.ymin) m.ymin = c[1];
    if (c[2] > m.zmax) m.zmax = c[2];
    if (c[2] < m.zmin) m.zmin = c[2];
    m.points.push_back({c[0], c[1], c[2]});
  }
  if (type == "SIZE") {
    m.size = num(value, kGeoErr, line);
    m.size_set = true;
  }
  if (type == "TYPE_DOMAIN") {
    if (value == "2D") m.is3d = false;
    else if (value == "3D") m.is3d = true;
  }
}

// GeometryReader::getCDWData (reader.cpp:832-958)
void geo_cdw(Mesh& m, const std::string& key, const std::string& value, unsigned line) {
  const std::string d = before(key, '(');
  if (d == "INITIAL_POSITION_SHAPES" || d == "END_POSITION_SHAPES") {
    int v = 0;
    if (!parse_int(value, v)) fail(fmt_line(kGeoErr, "The numeration of the point in the line %d is invalid", line));
    const uint32_t idx = (uint32_t)(v - 1);  // stored unsigned: 0 wraps to a huge index
    const uint32_t count = (uint32_t)m.points.size();
    if (d == "INITIAL_POSITION_SHAPES") {
      if (idx >= count)
        fail(fmt_line(kGeoErr, "The numeration of the point in the line %d doesn't exist or it can't be the last point",
                      line));
      m.idx_init = idx;
    } else {
      // the reference accepts idx == count and then reads past its point list
      if (idx >= count) fail(fmt_line(kGeoErr, "The numeration of the point in the line %d doesn't exist", line));
      m.idx_end = idx;
    }
  } else if (d == "CDW") {
    const int n = element_number(key, line);
    const bool exist = n <= (int)m.cdws.size();
    const std::string attr = attribute_after(key, ')', line);
    if (attr == "type") {
      if (exist) fail(fmt_line(kGeoErr, "The numeration of the CDW in the line %d already exist", line));
      if (value == "CIRCLE") m.cdws.push_back({CdwKind::Circle});
      else if (value == "RECTANGLE") m.cdws.push_back({CdwKind::Rectangle});
      else fail(fmt_line(kGeoErr, "The shape of the CDW in the line %d is not correct", line));
    } else if (attr == "height" || attr == "width" || attr == "radius") {
      if (!exist) fail("Error in the line " + std::to_string(line) + ". It is neccesary to specify the type of CDW first");
      Cdw& c = m.cdws[n - 1];
      const double v = num(value, kGeoErr, line);
      if (attr == "height" && c.kind == CdwKind::Rectangle) c.height = v;
      if (attr == "width" && c.kind == CdwKind::Rectangle) c.width = v;
      if (attr == "radius" && c.kind == CdwKind::Circle) c.radius = v;
    }
  }
  // SEPARATION is read by the reference but not used
}

// GeometryReader::getObstaclesData (reader.cpp:960-1124) and
// CalculationReader::getInitialConditions (reader.cpp:558-658) share the
// attribute handling; obstacles also take rotation, radius and thickness.
void shape_attribute(std::vector<Shape>& list, bool obstacle, const std::string& key, const std::string& value,
                     unsigned line, const char* prefix) {
  const int n = element_number(key, line);
  const bool exist = n <= (int)list.size();
  const std::string attr = attribute_after(key, ')', line);
  if (attr == "type") {
    if (exist) {
      if (obstacle) fail(fmt_line(prefix, "The numeration of the CDW in the line %d already exist", line));
      fail(fmt_line(prefix, "The initial condition in the line %d already exist", line));
    }
    if (obstacle && value == "WALL") list.emplace_back(ShapeKind::Rectangle);
    else if (obstacle && value == "CIRCLE") list.emplace_back(ShapeKind::Circle);
    else if (!obstacle && value == "CUBE") list.emplace_back(ShapeKind::Rectangle);
    else if (value == "CSV_2D") list.emplace_back(ShapeKind::Polygon);
    return;  // other values add nothing, as in the reference
  }
  static const char* known_obstacle[] = {"name", "position", "rotation", "height", "xWidth", "zWidth", "radius",
                                         "thickness"};
  static const char* known_initial[] = {"name", "position", "height", "xWidth", "zWidth"};
  bool known = false;
  if (obstacle) {
    for (const char* k : known_obstacle) known = known || attr == k;
  } else {
    for (const char* k : known_initial) known = known || attr == k;
  }
  if (!known) return;
  if (!exist) {
    if (obstacle)
      fail(fmt_line(prefix, "Error in the line %d. It is neccesary to specify the type of Obstacle first", line));
    fail(fmt_line(prefix, "Error in the line %d. It is neccesary to specify the type of initial condition first", line));
  }
  Shape& s = list[n - 1];
  if (attr == "name") {
    if (s.kind == ShapeKind::Polygon) s.filename = value + ".csv";
  } else if (attr == "position") {
    double c[3];
    triple(value, c, prefix, "position", line);
    s.set_position(c[0], c[1], c[2]);
  } else if (attr == "rotation") {
    double c[3];
    triple(value, c, prefix, "rotation", line);
    s.set_rotation(c[0] * kPi / 180.0, c[1] * kPi / 180.0, c[2] * kPi / 180.0);
  } else {
    const double v = num(value, prefix, line);
    if (s.kind == ShapeKind::Rectangle) {
      if (attr == "height") s.height = v;
      if (attr == "xWidth") s.xwidth = v;
      if (attr == "zWidth") s.zwidth = v;
    }
    if (s.kind == ShapeKind::Circle) {
      if (attr == "radius") s.radius = v;
      if (attr == "thickness") s.thickness = v;
    }
  }
}

void read_geometry(const std::string& path, Mesh& m) {
  std::ifstream in(path);
  if (!in.is_open()) fail("The file " + path + " cannot be opened", FLB_ERR_IO);
  std::string text;
  unsigned line = 0;
  while (std::getline(in, text)) {
    line++;
    std::string ns = text;
    ns.erase(std::remove(ns.begin(), ns.end(), ' '), ns.end());
    if ((!ns.empty() && ns[0] == '#') || text.empty()) continue;
    std::string key, value;
    if (!split_option(text, key, value)) fail(fmt_line(kGeoErr, "Error in the line %d", line));
    geo_mesh_elements(m, key, value, line);
    geo_cdw(m, key, value, line);
    if (before(key, '(') == "OBSTACLE") shape_attribute(m.obstacles, true, key, value, line, kGeoErr);
  }
  // GeometryReader::modifyGeometryData (reader.cpp:1126-1190), 2D part
  if (m.points.empty() || m.idx_init < 0 || m.idx_end < 0)
    fail(std::string(kGeoErr) + " POINT, INITIAL_POSITION_SHAPES and END_POSITION_SHAPES must be given");
  const double h_init = m.points[m.idx_init].y, h_end = m.points[m.idx_end].y;
  for (const Cdw& c : m.cdws) {
    double a = 0, b = 0;
    if (c.kind == CdwKind::Circle) {
      a = h_init + 2 * c.radius;
      b = h_end + 2 * c.radius;
    } else {
      a = h_init + c.height;
      b = h_end + c.height;
    }
    if (a > m.ymax) m.ymax = a;
    if (b > m.ymax) m.ymax = b;
  }
  const std::filesystem::path dir = std::filesystem::path(path).parent_path();
  for (Shape& s : m.obstacles) {
    if (s.kind == ShapeKind::Rectangle) s.init_rectangle();
    if (s.kind == ShapeKind::Polygon) s.init_polygon(dir.empty() ? std::filesystem::path(".") : dir);
  }
  // GeometryReader::checkOptionsGeometry (reader.cpp:766-774)
  if (m.idx_init >= m.idx_end)
    fail(std::string(kGeoErr) +
         " The numeration of the initial point of the geometry cannot be equal or greater than the end point");
  if (m.is3d) fail("TYPE_DOMAIN = 3D: the engine is two-dimensional (D2Q9)", FLB_ERR_UNSUPPORTED);
  if (!m.size_set || !(m.size > 0)) fail(std::string(kGeoErr) + " SIZE must be positive");
  // Mesh::calculateNumberPointsMesh (mesh.cpp:44-51)
  const double fx = std::floor((m.xmax - m.xmin) / m.size) + 1;
  const double fy = std::floor((m.ymax - m.ymin) / m.size) + 1;
  if (!(fx >= 1 && fy >= 1) || fx * fy > 4294967295.0 / 9.0)
    fail("the lattice of " + std::to_string(fx) + " x " + std::to_string(fy) + " cells is out of range",
         FLB_ERR_UNSUPPORTED);
  m.nx = (uint32_t)fx;
  m.ny = (uint32_t)fy;
  m.nz = 1;
}

uint8_t boundary_type(const std::string& v, uint8_t old) {
  if (v == "INPUT") return kInlet;
  if (v == "OUTPUT") return kOutlet;
  if (v == "WALL") return kWall;
  if (v == "PERIODIC") return kFluid;
  return old;
}

// CalculationReader::getOptionCalculation (reader.cpp:261-556).
void calc_option(Options& o, const std::string& key, std::string value, unsigned line) {
  bool bad = false;
  auto flag = [&](bool& dst) {
    if (value == "FALSE") dst = false;
    else if (value == "TRUE") dst = true;
    else bad = true;
  };
  auto positive_num = [&](const char* what) {
    double v = 0;
    if (!parse_double(value, v))
      fail(std::string(kCalcErr) + " The value of the " + what + " in the calculation's file in the line " +
           std::to_string(line) + " is invalid");
    return v;
  };
  if (key == "TYPE_ANALYSIS") {
    if (value == "2D") o.type_analysis = 0;
    else if (value == "3D") o.type_analysis = 1;
    else bad = true;
  } else if (key == "CALCULATION_API") {
    if (value != "CUDA") bad = true;
  } else if (key == "CUDA_BLOCK_SIZE") {
    std::string a, b, c;
    int v[3];
    if (!split_triple(value, a, b, c) || !parse_int(a, v[0]) || !parse_int(b, v[1]) || !parse_int(c, v[2]))
      fail(fmt_line(kCalcErr, "The value of the cuda block size in the line %d is invalid", line));
    for (int k = 0; k < 3; k++) o.block[k] = (uint32_t)v[k];
  } else if (key == "GRAPHICS_API") {
    if (value == "NONE") o.graphics = 0;
    else if (value == "OPENGL") o.graphics = 1;
    else bad = true;
  } else if (key == "TYPE_PROBLEM") {
    if (value == "MONOFLUID") o.free_surface = false;
    else if (value == "FREE_SURFACE") o.free_surface = true;
    else bad = true;
  } else if (key == "USE_VOLUMETRIC_FORCE") {
    flag(o.use_force);
  } else if (key == "ACCELERATION") {
    triple(value, o.acc, kCalcErr, "acceleration in the calculation's file", line);
  } else if (key == "VOLUMETRIC_FORCE") {
    triple(value, o.vforce, kCalcErr, "volumetric force in the calculation's file", line);
  } else if (key == "COLLISION_OPERATOR") {
    if (value == "SRT") o.collision = 0;
    else if (value == "TRT") o.collision = 1;
    else bad = true;
  } else if (key == "SUBGRID_TURBULENCE_MODEL") {
    flag(o.subgrid);
  } else if (key == "SURFACE_TENSION") {
    flag(o.surface_tension);
  } else if (key == "PRECISION") {
    if (value == "16") o.precision = 16;
    else if (value == "32") o.precision = 32;
    else if (value == "64") o.precision = 64;
    else bad = true;
  } else if (key == "REFERENCE_VELOCITY_LB" || key == "REFERENCE_VELOCITY_SI") {
    const double v = positive_num("reference velocity");
    if (key == "REFERENCE_VELOCITY_LB") o.ref_velocity_lb = v;
    else o.ref_velocity_si = v;
    if (v < 1e-6)
      fail(fmt_line(kCalcErr,
                    "The value of the reference velocity in the calculation's file in the line %d cannot be "
                    "negative or equal to zero",
                    line));
  } else if (key == "FLOW") {
    o.flow = positive_num("flow");
    if (o.flow < 0)
      fail(fmt_line(kCalcErr, "The value of the flow in the calculation's file in the line %d cannot be negative", line));
  } else if (key == "VELOCITY") {
    triple(value, o.vel_si, kCalcErr, "velocity in the calculation's file", line);
    if (o.vel_si[0] < 0 || o.vel_si[1] < 0 || o.vel_si[2] < 0)
      fail(fmt_line(kCalcErr, "The value of the velocity in the calculation's file in the line %d cannot be negative",
                    line));
  } else if (key == "RELAXATION_TIME") {
    o.relaxation_time = positive_num("relaxation time");
    if (o.relaxation_time <= 0.5)
      fail(fmt_line(kCalcErr,
                    "The value of the relaxation time in the calculation's file in the line %d must be greater than 0.5",
                    line));
  } else if (key == "KINEMATIC_VISCOSITY") {
    o.nu = positive_num("kinematic viscosity");
    if (o.nu < 0)
      fail(fmt_line(kCalcErr,
                    "The value of the kinematic viscosity in the calculation's file in the line %d cannot be negative",
                    line));
  } else if (key == "DENSITY") {
    o.density = positive_num("density");
    if (o.nu < 0)  // the reference tests the viscosity here; the density is checked at the end
      fail(fmt_line(kCalcErr, "The value of the density in the calculation's file in the line %d cannot be negative",
                    line));
  } else if (key == "LEFT_BOUNDARY") {
    o.left = boundary_type(value, o.left);
  } else if (key == "RIGHT_BOUNDARY") {
    o.right = boundary_type(value, o.right);
  } else if (key == "UP_BOUNDARY") {
    o.up = boundary_type(value, o.up);
  } else if (key == "DOWN_BOUNDARY") {
    o.down = boundary_type(value, o.down);
  } else if (key == "TIME_SIMULATION" || key == "TIME_SAVE") {
    float v = 0;
    if (!parse_float(value, v))
      fail(fmt_line(kCalcErr, "The value of the time in the calculation's file in the line %d is invalid", line));
    if (v < 0)
      fail(fmt_line(kCalcErr, "The value of the time in the calculation's file in the line %d cannot be negative", line));
    if (key == "TIME_SIMULATION") o.time_simulation = v;
    else o.time_save = v;
  } else if (key.substr(0, 7) != "INITIAL") {
    fail(fmt_line(kCalcErr, "The option in the calculation's file in the line %d doesn't exist", line));
  }
  if (bad) fail(fmt_line(kCalcErr, "The value of the option in the calculation's file in the line %d doesn't exist", line));
}

// CalculationReader::checkOptionsCalculation (reader.cpp:133-259).
void check_options(const Options& o, bool all) {
  auto zero = [](double v) { return std::abs(v - 0.0) <= 1e-6; };
  if (all && o.use_force &&
      zero(std::abs(o.vforce[0]) + std::abs(o.vforce[1]) + std::abs(o.vforce[2])) &&
      zero(std::abs(o.acc[0]) + std::abs(o.acc[1]) + std::abs(o.acc[2])))
    fail(std::string(kCalcErr) +
         " If volumetric forces are going to be used, some values of the forces themselves or the acceleration must "
         "be indicated");
  const double vsum = o.vel_si[0] + o.vel_si[1] + o.vel_si[2];
  if (all && o.flow > 1e-10 && vsum > 1e-10)
    fail(std::string(kCalcErr) + " Only one of the two arguments, flow and velocity, must be idicated, not both");
  if (all && o.flow < 1e-10 && vsum < 1e-10)
    fail(std::string(kCalcErr) + " One of the two arguments, flow or velocity, must be idicated");
  if (all && o.nu < 1e-12)
    fail(std::string(kCalcErr) + " The kinematic viscosity has to have a value or be positive");
  if (all && o.density < 1e-12) fail(std::string(kCalcErr) + " The density has to have a value or be positive");
  if (o.left == kNone) fail(std::string(kCalcErr) + " The boundary condition LEFT_BOUNDARY cannot be NONE");
  if (o.right == kNone) fail(std::string(kCalcErr) + " The boundary condition RIGHT_BOUNDARY cannot be NONE");
  if (o.up == kNone) fail(std::string(kCalcErr) + " The boundary condition UP_BOUNDARY cannot be NONE");
  if (o.down == kNone) fail(std::string(kCalcErr) + " The boundary condition DOWN_BOUNDARY cannot be NONE");
  if (o.left != o.right && (o.left & ~(kInlet | kWall)))
    fail(std::string(kCalcErr) +
         " The boundary conditions LEFT_BOUNDARY and RIGHT_BOUNDARY must be equal if a periodic boundary is selected");
  if (all) {
    if (o.block[0] == 0)
      fail(std::string(kCalcErr) +
           " The value of the cuda block size in the x direction cannot be negative or equal to zero");
    if (o.block[1] == 0)
      fail(std::string(kCalcErr) +
           " The value of the cuda block size in the y direction cannot be negative or equal to zero");
    const uint32_t threads = o.block[0] * o.block[1];
    if (o.type_analysis == 0 && threads > kMaxThreadsPerBlock)
      fail(std::string(kCalcErr) + " The threads per block is superior to the maximum, " + std::to_string(threads) +
           " > " + std::to_string(kMaxThreadsPerBlock));
  }
  if (all && o.graphics == 0) {
    if (std::abs(o.time_save - 0.0f) <= 1e-6f) fail(std::string(kCalcErr) + " The save time cannot be 0");
    if (std::abs(o.time_simulation - 0.0f) <= 1e-6f) fail(std::string(kCalcErr) + " The simulation time cannot be 0");
    if (o.time_save >= o.time_simulation) {
      char b[160];
      std::snprintf(b, sizeof b, " The save time is greater than the simulation time, %6.4f > %6.4f",
                    (double)o.time_save, (double)o.time_simulation);
      fail(std::string(kCalcErr) + b);
    }
  }
}

void read_options(const std::string& path, Options& o, Mesh& m, bool mesh_only) {
  std::ifstream in(path);
  if (!in.is_open()) fail("The file " + path + " cannot be opened", FLB_ERR_IO);
  static const char* mesh_keys[] = {"TYPE_PROBLEM", "LEFT_BOUNDARY", "RIGHT_BOUNDARY", "UP_BOUNDARY", "DOWN_BOUNDARY"};
  std::string text;
  unsigned line = 0;
  while (std::getline(in, text)) {
    line++;
    if (mesh_only) {  // readSomeOptionsCalculation removes the spaces first (reader.cpp:715-742)
      text.erase(std::remove(text.begin(), text.end(), ' '), text.end());
      if ((!text.empty() && text[0] == '#') || text.empty()) continue;
    } else {
      std::string ns = text;
      ns.erase(std::remove(ns.begin(), ns.end(), ' '), ns.end());
      if ((!ns.empty() && ns[0] == '#') || text.empty()) continue;
    }
    std::string key, value;
    if (!split_option(text, key, value)) fail(fmt_line(kCalcErr, "Error in the line %d", line));
    const bool is_initial = before(key, '(') == "INITIAL_CONDITION_FLAG";
    if (mesh_only) {
      if (is_initial) shape_attribute(m.initial, false, key, value, line, kCalcErr);
      bool listed = false;
      for (const char* k : mesh_keys) listed = listed || key == k;
      if (listed) calc_option(o, key, value, line);
    } else {
      calc_option(o, key, value, line);
      if (is_initial) shape_attribute(m.initial, false, key, value, line, kCalcErr);
    }
  }
  const std::filesystem::path dir = std::filesystem::path(path).parent_path();
  for (Shape& s : m.initial) {
    if (s.kind == ShapeKind::Rectangle) s.init_rectangle();
    if (s.kind == ShapeKind::Polygon) s.init_polygon(dir.empty() ? std::filesystem::path(".") : dir);
  }
  check_options(o, !mesh_only);
  if (!mesh_only && o.type_analysis == 1)
    fail("TYPE_ANALYSIS = 3D: the engine is two-dimensional (D2Q9)", FLB_ERR_UNSUPPORTED);
}

// getEndPointBaseCoordinate (initData.h:42-53): index of the first point
// after the first whose x reaches xSI.  The reference can return the point
// count (a node right of every point) and then reads past its list; this
// clamps to the last point.
uint32_t end_point_base(double x, const std::vector<Point>& p) {
  uint32_t c = 1;
  for (size_t i = 1; i < p.size(); i++) {
    if (p[i].x >= (x - 1e-12)) return c;
    c++;
  }
  return (uint32_t)p.size() - 1;
}

// The geometry sweep of initData (initData.h:220-317).
void sweep_flags(const Mesh& m, const Options& o, uint8_t* flags) {
  const double eps = kEps;
  const std::vector<Point>& p = m.points;
  const double ix = p[m.idx_init].x - eps, ex = p[m.idx_end].x + eps;
  const uint8_t dflt = o.free_surface ? kGas : kFluid;
  for (uint32_t y = 0; y < m.ny; y++) {
    for (uint32_t x = 0; x < m.nx; x++) {
      const uint32_t idx = x + y * m.nx;
      uint8_t f = (uint8_t)idx;  // h_flags.push_back(idx): a node no rule reaches keeps this byte
      const double xs = m.xmin + x * m.size, ys = m.ymin + y * m.size, zs = m.zmin + 0 * m.size;
      const uint32_t b = end_point_base(xs, p);
      const double slope = (p[b].y - p[b - 1].y) / (p[b].x - p[b - 1].x);
      const double base = p[b - 1].y + (xs - p[b - 1].x) * slope;
      if (xs >= ix && xs <= ex) {
        for (const Cdw& c : m.cdws) f = c.inside(xs, ys, zs, p, b) ? dflt : kWall;
      } else {
        if (ys <= (base + eps)) f = o.down;
        else if (ys >= (m.ymax - eps)) f = o.up;
      }
      if (ys <= (base + eps) && f == dflt) f = o.down;
      else if (ys >= (m.ymax - eps) && f == dflt) f = o.up;
      else if (x == 0 && f == dflt) f = o.left;
      else if (x == (m.nx - 1) && f == dflt) f = o.right;
      for (const Shape& s : m.obstacles)
        if (s.inside(xs, ys, zs)) f = kWall;
      for (const Shape& s : m.initial)
        if (s.inside(xs, ys, zs)) f = kFluid;
      flags[idx] = f;
    }
  }
}

// initFreeSurfaceFlags (initData.cpp:13-37) over all cells in index order:
// inlet cells gain the FLUID bit, outlet cells the GAS bit, and GAS
// neighbours (non-periodic, eight directions) of FLUID cells become INTERFACE.
void sweep_free_surface(uint8_t* flags, uint32_t nx, uint32_t ny) {
  for (uint32_t y = 0; y < ny; y++) {
    for (uint32_t x = 0; x < nx; x++) {
      uint8_t& f = flags[x + y * nx];
      if (f & ~(kFluid | kInlet | kOutlet)) continue;
      if (f & kInlet) f |= kFluid;
      else if (f & kOutlet) f |= kGas;
      if (!(f & kFluid)) continue;
      for (int dy = -1; dy <= 1; dy++) {
        for (int dx = -1; dx <= 1; dx++) {
          if (!dx && !dy) continue;
          const long xx = (long)x + dx, yy = (long)y + dy;
          if (xx < 0 || yy < 0 || xx >= (long)nx || yy >= (long)ny) continue;
          uint8_t& g = flags[(size_t)xx + (size_t)yy * nx];
          if (g == kGas) g = kInterface;
        }
      }
    }
  }
}

// Units::setConversionParameters and the conversions (utils.cpp:7-82),
// then h_initConstantDataCuda2D's tau and force (cudaInitData.cu:57-82) and
// the loop bounds of the headless loops (runCuda.cu:462-464, 497-499).
void derive(const Mesh& m, const Options& o, flb_setup* s) {
  const double length = m.xmax - m.xmin, lb_length = (double)(m.nx - 1);
  const double L = length / lb_length;
  const double T = L * o.ref_velocity_lb / o.ref_velocity_si;
  const double M = o.density / 1.0 * (L * L * L);
  s->length_to_si = L;
  s->time_to_si = T;
  s->mass_to_si = M;
  s->velocity_to_si = L / T;
  s->rho_to_si = M / (L * L * L);
  const double vlb[2] = {o.vel_si[0] / (L / T), o.vel_si[1] / (L / T)};
  const bool has_tau = !(std::abs(o.relaxation_time - 0.0) <= 1e-6);
  float nu = 0.0f;
  if (has_tau) nu = (float)((o.relaxation_time - 0.5) / 3.0);
  else nu = (float)((double)(float)o.nu * T / (L * L));
  auto force = [&](double acc, double vf) -> float {
    if (std::abs(acc - 0.0) <= 1e-6) return (float)(vf * T * T * L * L / M);
    return (float)(o.density * acc * L * L * T * T / M);
  };
  float fx = 0.0f, fy = 0.0f;
  if (o.use_force) {
    fx = force(o.acc[0], o.vforce[0]);
    fy = force(o.acc[1], o.vforce[1]);
  }
  const float tau = has_tau ? (float)o.relaxation_time : 3.0f * nu + 0.5f;
  auto to_lattice_steps = [&](float t_si) -> uint64_t {
    const float v = (float)((double)t_si / T);
    return (v >= 0.0f && std::isfinite(v)) ? (uint64_t)v : 0;
  };
  s->time_steps = to_lattice_steps(o.time_simulation);
  s->save_every = to_lattice_steps(o.time_save);
  s->time_simulation = o.time_simulation;
  s->time_save = o.time_save;
  s->nu_lattice = nu;

  flb_case_desc& d = s->desc;
  flb_case_desc_init(&d);
  d.nx = m.nx;
  d.ny = m.ny;
  d.flags = s->flags;
  d.free_surface = o.free_surface ? 1 : 0;
  d.precision = o.precision;
  d.mass_precision = o.precision == 32 ? 32 : 64;
  d.collision = o.collision;
  d.subgrid = o.subgrid ? 1 : 0;
  d.use_volumetric_force = o.use_force ? 1 : 0;
  d.tau = tau;
  d.fx = fx;
  d.fy = fy;
  d.inlet_ux = vlb[0];
  d.inlet_uy = vlb[1];
  d.bounce_back = FLB_BB_IMPLICIT;
  d.fs_mode = FLB_FS_REFERENCE;
  d.arithmetic = FLB_ARITH_REFERENCE;
}

void set_error(flb_setup* s, const std::string& msg) {
  if (!s) return;
  std::snprintf(s->error, sizeof s->error, "%s", msg.c_str());
}

// ---- VTK ImageData writer (io/writer.cpp) --------------------------------

// Values are written as the reference's std::ostream does with its default
// format, which is printf's %g.
void put_g(std::string& out, double v) {
  char b[64];
  std::snprintf(b, sizeof b, "%g", v);
  out += b;
}

std::string f6(double v) {
  char b[64];
  std::snprintf(b, sizeof b, "%f", v);  // std::to_string(double)
  return b;
}

double value_at(const flb_vti_field& f, size_t i) {
  switch (f.type) {
    case FLB_VTI_UINT8: return (double)(int)((const uint8_t*)f.data)[i];
    case FLB_VTI_FLOAT32: return (double)((const float*)f.data)[i];
    default: return ((const double*)f.data)[i];
  }
}

const char* type_name(int t) {
  switch (t) {
    case FLB_VTI_UINT8: return "UInt8";
    case FLB_VTI_FLOAT32: return "Float32";
    case FLB_VTI_FLOAT64: return "Float64";
    default: return nullptr;
  }
}

flb_status write_vti(const char* path, uint32_t nx, uint32_t ny, double x0, double y0, double z0, double spacing,
                     const flb_vti_field* fields, uint32_t n_fields) {
  if (!path || nx == 0 || ny == 0 || (n_fields && !fields)) return FLB_ERR_INVALID_ARGUMENT;
  const size_t N = (size_t)nx * ny;
  for (uint32_t k = 0; k < n_fields; k++) {
    const flb_vti_field& f = fields[k];
    if (!f.name || !f.data || !type_name(f.type) || (f.components != 1 && f.components != 2 && f.components != 3))
      return FLB_ERR_INVALID_ARGUMENT;
  }
  std::FILE* fp = std::fopen(path, "wb");
  if (!fp) return FLB_ERR_IO;
  const std::string extent = "0 " + std::to_string(nx - 1) + " 0 " + std::to_string(ny - 1) + " 0 0";
  std::string out;
  out.reserve(1 << 20);
  out += "<VTKFile type=\"ImageData\" version=\"1.0\">\n";
  out += "<ImageData WholeExtent=\"" + extent + "\" Origin=\"" + f6(x0) + " " + f6(y0) + " " + f6(z0) +
         "\" Spacing=\"" + f6(spacing) + " " + f6(spacing) + " " + f6(spacing) + "\" >\n";
  out += "<Piece Extent=\"" + extent + "\" >\n";
  out += "<PointData>\n";
  bool ok = true;
  auto flush = [&]() {
    if (!out.empty() && std::fwrite(out.data(), 1, out.size(), fp) != out.size()) ok = false;
    out.clear();
  };
  for (uint32_t k = 0; k < n_fields && ok; k++) {
    const flb_vti_field& f = fields[k];
    out += std::string("<DataArray type=\"") + type_name(f.type) + "\" Name=\"" + f.name +
           "\" NumberOfComponents=\"" + std::to_string(f.components) + "\" format=\"ascii\">\n";
    const double ysign = f.flip_y ? -1.0 : 1.0;
    for (size_t i = 0; i < N; i++) {
      if (f.components == 1) {
        put_g(out, value_at(f, i) * f.to_si);
        out += "\n";
      } else {
        put_g(out, value_at(f, i) * f.to_si);
        out += " ";
        put_g(out, value_at(f, i + N) * f.to_si * ysign);
        if (f.components == 3) {
          out += " ";
          put_g(out, value_at(f, i + 2 * N) * f.to_si);
        }
        out += "\n";
      }
      if (out.size() > (1u << 20)) flush();
    }
    out += "</DataArray>\n";
  }
  out += "</PointData>\n<CellData>\n</CellData>\n</Piece>\n</ImageData>\n</VTKFile>\n";
  flush();
  if (std::fclose(fp) != 0) ok = false;
  return ok ? FLB_OK : FLB_ERR_IO;
}

flb_status write_series(const char* directory, uint32_t n_files, double dt) {
  if (!directory) return FLB_ERR_INVALID_ARGUMENT;
  const std::string path = (std::filesystem::path(directory) / "loaderFiles.vti.series").string();
  std::FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) return FLB_ERR_IO;
  std::string out = "{\n\"file-series-version\" : \"1.0\",\n\"files\" : [\n";
  for (uint32_t i = 0; i < n_files; i++)
    out += "{\"name\" : \"result_" + std::to_string(i) + ".vti\", \"time\" : " + f6((double)i * dt) + "},\n";
  out += "]\n}";
  const bool ok = std::fwrite(out.data(), 1, out.size(), fp) == out.size();
  return (std::fclose(fp) == 0 && ok) ? FLB_OK : FLB_ERR_IO;
}

}  // namespace

extern "C" {

FLB_API flb_status flb_setup_from_files(const char* geometry_txt, const char* options_txt, int mesh_only,
                                        flb_setup* out) {
  if (!out) return FLB_ERR_INVALID_ARGUMENT;
  std::memset(out, 0, sizeof(*out));
  if (!geometry_txt || !options_txt) {
    set_error(out, "geometry and options paths are required");
    return FLB_ERR_INVALID_ARGUMENT;
  }
  try {
    Mesh m;
    Options o;
    read_geometry(geometry_txt, m);
    read_options(options_txt, o, m, mesh_only != 0);
    const size_t N = (size_t)m.nx * m.ny;
    out->flags = (uint8_t*)std::malloc(N);
    if (!out->flags) fail("out of host memory for the flags", FLB_ERR_OUT_OF_MEMORY);
    sweep_flags(m, o, out->flags);
    out->nx = m.nx;
    out->ny = m.ny;
    out->x_min = m.xmin;
    out->y_min = m.ymin;
    out->z_min = m.zmin;
    out->spacing = m.size;
    out->graphics_api = o.graphics;
    out->reference_precision = o.precision;
    for (int k = 0; k < 3; k++) out->cuda_block[k] = o.block[k];
    if (mesh_only) {
      flb_case_desc_init(&out->desc);
      out->desc.nx = m.nx;
      out->desc.ny = m.ny;
      out->desc.flags = out->flags;
      out->desc.free_surface = o.free_surface ? 1 : 0;
    } else {
      derive(m, o, out);
    }
  } catch (const SetupError& e) {
    std::free(out->flags);
    out->flags = nullptr;
    out->desc.flags = nullptr;
    set_error(out, e.msg);
    return e.status;
  } catch (const std::exception& e) {
    std::free(out->flags);
    out->flags = nullptr;
    out->desc.flags = nullptr;
    set_error(out, e.what());
    return FLB_ERR_INVALID_ARGUMENT;
  }
  return FLB_OK;
}

FLB_API void flb_setup_free(flb_setup* s) {
  if (!s) return;
  std::free(s->flags);
  s->flags = nullptr;
  s->desc.flags = nullptr;
}

FLB_API flb_status flb_setup_initial_flags(const flb_setup* s, uint8_t* out) {
  if (!s || !s->flags || !out) return FLB_ERR_INVALID_ARGUMENT;
  const size_t N = (size_t)s->nx * s->ny;
  std::memcpy(out, s->flags, N);
  if (s->desc.free_surface) sweep_free_surface(out, s->nx, s->ny);
  return FLB_OK;
}

FLB_API flb_status flb_setup_write_mesh_vti(const flb_setup* s, const char* path) {
  if (!s || !s->flags || !path) return FLB_ERR_INVALID_ARGUMENT;
  std::vector<uint8_t> f((size_t)s->nx * s->ny);
  flb_status st = flb_setup_initial_flags(s, f.data());
  if (st != FLB_OK) return st;
  flb_vti_field field{};
  field.name = "Flags";
  field.type = FLB_VTI_UINT8;
  field.components = 1;
  field.data = f.data();
  field.to_si = 1.0;
  return write_vti(path, s->nx, s->ny, s->x_min, s->y_min, s->z_min, s->spacing, &field, 1);
}

FLB_API flb_status flb_create_from_files(const char* geometry_txt, const char* options_txt, flb_handle* out) {
  if (!out) return FLB_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  flb_setup s;
  flb_status st = flb_setup_from_files(geometry_txt, options_txt, 0, &s);
  if (st != FLB_OK) {
    std::fprintf(stderr, "flb_create_from_files: %s\n", s.error);
    return st;
  }
  st = flb_create(&s.desc, out);
  flb_setup_free(&s);
  return st;
}

FLB_API flb_status flb_write_vti(const char* path, uint32_t nx, uint32_t ny, double x0, double y0, double z0,
                                 double spacing, const flb_vti_field* fields, uint32_t n_fields) {
  return write_vti(path, nx, ny, x0, y0, z0, spacing, fields, n_fields);
}

FLB_API flb_status flb_write_vti_series(const char* directory, uint32_t n_files, double time_interval) {
  return write_series(directory, n_files, time_interval);
}

FLB_API flb_status flb_run_from_files(const char* geometry_txt, const char* options_txt, const char* save_dir,
                                      uint64_t max_steps, flb_run_info* info) {
  if (info) std::memset(info, 0, sizeof(*info));
  flb_setup s;
  flb_status st = flb_setup_from_files(geometry_txt, options_txt, 0, &s);
  if (st != FLB_OK) {
    if (info) std::snprintf(info->error, sizeof info->error, "%s", s.error);
    return st;
  }
  auto finish = [&](flb_status r, const char* msg) {
    if (info && msg) std::snprintf(info->error, sizeof info->error, "%s", msg);
    flb_setup_free(&s);
    return r;
  };
  if (!save_dir) return finish(FLB_ERR_INVALID_ARGUMENT, "save_dir is required");
  if (s.save_every == 0) return finish(FLB_ERR_INVALID_ARGUMENT, "TIME_SAVE is shorter than one lattice time step");
  // VTIWriter's constructor: a new folder results_<i> (writer.cpp:199-212)
  std::filesystem::path dir;
  try {
    int i = 0;
    do {
      dir = std::filesystem::path(save_dir) / ("results_" + std::to_string(i++));
    } while (std::filesystem::exists(dir));
    if (!std::filesystem::create_directories(dir)) return finish(FLB_ERR_IO, "cannot create the results folder");
  } catch (const std::exception& e) {
    return finish(FLB_ERR_IO, e.what());
  }
  if (info) std::snprintf(info->directory, sizeof info->directory, "%s", dir.string().c_str());
  flb_handle h = nullptr;
  st = flb_create(&s.desc, &h);
  if (st != FLB_OK) return finish(st, "flb_create failed");
  const size_t N = (size_t)s.nx * s.ny;
  size_t esize = 0, count = 0;
  flb_field_info(h, FLB_FIELD_RHO, &esize, &count);
  const int ftype = esize == 8 ? FLB_VTI_FLOAT64 : FLB_VTI_FLOAT32;
  size_t msize = 0, mcount = 0;
  if (s.desc.free_surface) flb_field_info(h, FLB_FIELD_PHI, &msize, &mcount);
  std::vector<unsigned char> u(2 * N * esize), rho(N * esize), phi(N * (msize ? msize : 1));
  std::vector<uint8_t> flags(N);
  const uint64_t total = s.time_steps + 1;  // while (t <= timeSimulation)
  const uint64_t steps = max_steps ? std::min<uint64_t>(max_steps, total) : total;
  uint64_t t = 0;
  uint32_t files = 0;
  while (t < steps && st == FLB_OK) {
    // the step with index t is followed by a save when t % tSave == 0
    const uint64_t to_save = (t % s.save_every == 0) ? t : (t / s.save_every + 1) * s.save_every;
    const uint64_t n = std::min<uint64_t>(to_save - t + 1, steps - t);
    st = flb_step(h, n);
    if (st != FLB_OK) break;
    t += n;
    if ((t - 1) % s.save_every != 0) continue;
    st = flb_read_field(h, FLB_FIELD_U, u.data(), 0);
    if (st == FLB_OK) st = flb_read_field(h, FLB_FIELD_RHO, rho.data(), 0);
    if (st == FLB_OK) st = flb_read_field(h, FLB_FIELD_FLAGS, flags.data(), 0);
    if (st == FLB_OK && s.desc.free_surface) st = flb_read_field(h, FLB_FIELD_PHI, phi.data(), 0);
    if (st != FLB_OK) break;
    // runCuda.cu:480-484 (mono-fluid, SI units) and :516-521 (free surface, lattice units)
    const double uc = s.desc.free_surface ? 1.0 : s.velocity_to_si;
    const double rc = s.desc.free_surface ? 1.0 : s.rho_to_si;
    flb_vti_field fl[4] = {};
    fl[0] = {"Flags", FLB_VTI_UINT8, 1, flags.data(), 1.0, 0};
    fl[1] = {"U", ftype, 2, u.data(), uc, 0};
    fl[2] = {"rho", ftype, 1, rho.data(), rc, 0};
    fl[3] = {"phi", msize == 8 ? FLB_VTI_FLOAT64 : FLB_VTI_FLOAT32, 1, phi.data(), 1.0, 0};
    const std::string file = (dir / ("result_" + std::to_string(files) + ".vti")).string();
    st = write_vti(file.c_str(), s.nx, s.ny, s.x_min, s.y_min, s.z_min, s.spacing, fl, s.desc.free_surface ? 4 : 3);
    if (st != FLB_OK) break;
    files++;
    st = write_series(dir.string().c_str(), files, (double)s.time_save);
  }
  if (info) {
    info->steps = t;
    info->files = files;
  }
  flb_destroy(h);
  return finish(st, st == FLB_OK ? nullptr : "the run stopped on an error");
}

}  // extern "C"
