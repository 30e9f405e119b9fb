// PLY textured meshes, as ReadTexturedMesh / WriteTexturedMesh read and write
// them (include/Src/SimpleMesh.h:93-160).  Item conversion follows the
// reference's PLY library (include/Misha/PlyFile.inl:2342-2560): ASCII
// integers through atoi (unsigned through strtol), ASCII reals through atof
// straight to double (a "float" column is not rounded to float32), binary
// items in their declared type, byte-swapped when the file's endianness is not
// the machine's, then widened.
#include "io/texture_io.h"

#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <sstream>
#include <utility>

namespace gdtp {
namespace io {
namespace {

enum PlyType { kNone = -1, kI8, kU8, kI16, kU16, kI32, kU32, kF32, kF64 };

PlyType ply_type(const std::string& s) {
  if (s == "char" || s == "int8") return kI8;
  if (s == "uchar" || s == "uint8") return kU8;
  if (s == "short" || s == "int16") return kI16;
  if (s == "ushort" || s == "uint16") return kU16;
  if (s == "int" || s == "int32") return kI32;
  if (s == "uint" || s == "uint32") return kU32;
  if (s == "float" || s == "float32") return kF32;
  if (s == "double" || s == "float64") return kF64;
  return kNone;
}
int type_size(PlyType t) { return t == kI8 || t == kU8 ? 1 : t == kI16 || t == kU16 ? 2 : t == kF64 ? 8 : 4; }

struct Property {
  std::string name;
  PlyType type = kNone, countType = kNone;  // countType != kNone: a list
};
struct Element {
  std::string name;
  long long count = 0;
  std::vector<Property> props;
};

// One item: its int, unsigned and double readings, as the reference's
// get_ascii_item / get_binary_item produce them
struct Item {
  int i = 0;
  unsigned u = 0;
  double d = 0;
  // a real's integer readings; values outside the integer range (undefined
  // behaviour in the reference) read as 0
  void from_real(double v) {
    d = v;
    i = v > -2147483649.0 && v < 2147483648.0 ? int(v) : 0;
    u = v > -1.0 && v < 4294967296.0 ? unsigned(v) : 0u;
  }
};

class Reader {
 public:
  Reader(const std::vector<char>& buf, size_t pos, int format) : b_(buf), p_(pos), fmt_(format) {}
  bool next(PlyType t, Item& it) {
    if (fmt_ == 0) return ascii(t, it);
    const int n = type_size(t);
    if (p_ + n > b_.size()) return false;
    unsigned char c[8];
    std::memcpy(c, b_.data() + p_, n);
    p_ += n;
    const bool little = fmt_ == 1;
    const uint16_t probe = 1;
    const bool hostLittle = *reinterpret_cast<const unsigned char*>(&probe) == 1;
    if (little != hostLittle)
      for (int k = 0; k < n / 2; k++) std::swap(c[k], c[n - 1 - k]);
    switch (t) {
      case kI8: { signed char v; std::memcpy(&v, c, 1); it.i = v, it.u = unsigned(it.i), it.d = it.i; break; }
      case kU8: { it.u = c[0], it.i = int(it.u), it.d = it.u; break; }
      case kI16: { int16_t v; std::memcpy(&v, c, 2); it.i = v, it.u = unsigned(it.i), it.d = it.i; break; }
      case kU16: { uint16_t v; std::memcpy(&v, c, 2); it.u = v, it.i = int(it.u), it.d = it.u; break; }
      case kI32: { int32_t v; std::memcpy(&v, c, 4); it.i = v, it.u = unsigned(it.i), it.d = it.i; break; }
      case kU32: { uint32_t v; std::memcpy(&v, c, 4); it.u = v, it.i = int(it.u), it.d = it.u; break; }
      case kF32: { float v; std::memcpy(&v, c, 4); it.from_real(v); break; }
      case kF64: { double v; std::memcpy(&v, c, 8); it.from_real(v); break; }
      default: return false;
    }
    return true;
  }

 private:
  bool ascii(PlyType t, Item& it) {
    while (p_ < b_.size() && std::isspace(static_cast<unsigned char>(b_[p_]))) p_++;
    if (p_ >= b_.size()) return false;
    const size_t s = p_;
    while (p_ < b_.size() && !std::isspace(static_cast<unsigned char>(b_[p_]))) p_++;
    word_.assign(b_.data() + s, p_ - s);
    const char* w = word_.c_str();
    if (t == kU32) {
      it.u = unsigned(std::strtol(w, nullptr, 10)), it.i = int(it.u), it.d = it.u;
    } else if (t == kF32 || t == kF64) {
      it.from_real(std::atof(w));
    } else {
      it.i = std::atoi(w), it.u = unsigned(it.i), it.d = it.i;
    }
    return true;
  }
  const std::vector<char>& b_;
  size_t p_;
  int fmt_;  // 0 ascii, 1 binary little endian, 2 binary big endian
  std::string word_;
};

}  // namespace

bool read_ply_textured_mesh(const std::string& path, TexturedMesh& m, std::string& err) {
  std::ifstream f(path, std::ios::binary);
  if (!f) { err = "cannot open " + path; return false; }
  std::vector<char> buf((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  // header: lines up to "end_header"
  size_t pos = 0;
  auto line = [&](std::string& out) {
    if (pos >= buf.size()) return false;
    size_t e = pos;
    while (e < buf.size() && buf[e] != '\n') e++;
    out.assign(buf.data() + pos, e - pos);
    if (!out.empty() && out.back() == '\r') out.pop_back();
    pos = e < buf.size() ? e + 1 : e;
    return true;
  };
  std::string l;
  if (!line(l) || l != "ply") { err = path + ": not a PLY file"; return false; }
  int format = -1;
  std::vector<Element> elems;
  m = TexturedMesh();
  bool ended = false;
  while (line(l)) {
    std::istringstream ss(l);
    std::string kw;
    ss >> kw;
    if (kw == "format") {
      std::string f1;
      ss >> f1;
      format = f1 == "ascii" ? 0 : f1 == "binary_little_endian" ? 1 : f1 == "binary_big_endian" ? 2 : -1;
      if (format < 0) { err = path + ": unknown PLY format " + f1; return false; }
    } else if (kw == "comment") {
      std::string tag, name;
      ss >> tag;
      if (tag == "TextureFile") {
        std::getline(ss, name);
        const size_t a = name.find_first_not_of(" \t");
        m.textureFile = a == std::string::npos ? "" : name.substr(a);
      }
    } else if (kw == "element") {
      Element e;
      ss >> e.name >> e.count;
      if (e.name.empty() || e.count < 0) { err = path + ": bad PLY element line"; return false; }
      elems.push_back(e);
    } else if (kw == "property") {
      if (elems.empty()) { err = path + ": PLY property before any element"; return false; }
      std::string t1;
      ss >> t1;
      Property p;
      if (t1 == "list") {
        std::string ct, it;
        ss >> ct >> it >> p.name;
        p.countType = ply_type(ct), p.type = ply_type(it);
        if (p.countType == kNone || p.type == kNone || p.countType == kF32 || p.countType == kF64) {
          err = path + ": bad PLY list property " + p.name;
          return false;
        }
      } else {
        p.type = ply_type(t1);
        ss >> p.name;
        if (p.type == kNone) { err = path + ": unknown PLY type " + t1; return false; }
      }
      elems.back().props.push_back(p);
    } else if (kw == "end_header") {
      ended = true;
      break;
    } else if (kw.empty() || kw == "obj_info") {
      continue;
    } else {
      err = path + ": unexpected PLY header line: " + l;
      return false;
    }
  }
  if (!ended || format < 0) { err = path + ": incomplete PLY header"; return false; }
  // every instance takes at least its scalars and list counts (binary) or one
  // character and a separator per item (ASCII): counts the file cannot hold are
  // rejected before anything is allocated for them
  {
    long double need = 0;
    for (const Element& e : elems) {
      long double per = 0;
      for (const Property& p : e.props) per += format == 0 ? 2 : type_size(p.countType != kNone ? p.countType : p.type);
      need += per * (long double)e.count;
    }
    if (need > (long double)(buf.size() - pos)) { err = path + ": PLY element counts exceed the file size"; return false; }
  }

  Reader r(buf, pos, format);
  Item it;
  bool haveVertices = false, haveFaces = false;
  for (const Element& e : elems) {
    const bool isVertex = e.name == "vertex", isFace = e.name == "face";
    int xyz[3] = {-1, -1, -1}, vidx = -1, tex = -1;
    for (size_t k = 0; k < e.props.size(); k++) {
      const std::string& n = e.props[k].name;
      if (isVertex && e.props[k].countType == kNone) {
        if (n == "x") xyz[0] = int(k);
        if (n == "y") xyz[1] = int(k);
        if (n == "z") xyz[2] = int(k);
      }
      if (isFace && e.props[k].countType != kNone) {
        if (n == "vertex_indices" || (n == "vertex_index" && vidx < 0)) vidx = int(k);
        if (n == "texcoord") tex = int(k);
      }
    }
    if (isVertex) {
      if (xyz[0] < 0 || xyz[1] < 0 || xyz[2] < 0) { err = path + ": vertices without x, y, z"; return false; }
      m.vertices.assign(size_t(e.count) * 3, 0.0);
      haveVertices = true;
    }
    if (isFace) {
      if (vidx < 0) { err = path + ": faces without vertex_indices"; return false; }
      if (tex < 0) { err = path + ": faces without texcoord (not a textured mesh)"; return false; }
      m.triangles.assign(size_t(e.count) * 3, 0);
      m.uv.assign(size_t(e.count) * 6, 0.0);
      haveFaces = true;
    }
    for (long long i = 0; i < e.count; i++) {
      for (size_t k = 0; k < e.props.size(); k++) {
        const Property& p = e.props[k];
        if (p.countType == kNone) {
          if (!r.next(p.type, it)) { err = path + ": PLY data ends early"; return false; }
          if (isVertex)
            for (int c = 0; c < 3; c++)
              if (xyz[c] == int(k)) m.vertices[3 * size_t(i) + c] = it.d;
          continue;
        }
        if (!r.next(p.countType, it)) { err = path + ": PLY data ends early"; return false; }
        const int cnt = it.i;
        if (cnt < 0) { err = path + ": negative PLY list length"; return false; }
        const bool isIdx = isFace && int(k) == vidx, isTex = isFace && int(k) == tex;
        if (isIdx && cnt < 3) { err = path + ": face " + std::to_string(i) + " has fewer than 3 corners"; return false; }
        if (isTex && cnt < 6) { err = path + ": face " + std::to_string(i) + " has fewer than 3 texture coordinates"; return false; }
        for (int j = 0; j < cnt; j++) {
          if (!r.next(p.type, it)) { err = path + ": PLY data ends early"; return false; }
          if (isIdx && j < 3) m.triangles[3 * size_t(i) + j] = it.i;
          if (isTex && j < 6) m.uv[6 * size_t(i) + j] = it.d;
        }
      }
    }
  }
  if (!haveVertices || !haveFaces) { err = path + ": PLY has no vertex or no face element"; return false; }
  const long long nv = (long long)m.vertices.size() / 3;
  for (int t : m.triangles)
    if (t < 0 || t >= nv) { err = path + ": face refers to a vertex out of range"; return false; }
  return true;
}

bool write_ply_textured_mesh(const std::string& path, const TexturedMesh& m, std::string& err) {
  if (m.vertices.size() % 3 || m.triangles.size() % 3 || m.uv.size() != m.triangles.size() * 2) {
    err = "inconsistent textured mesh arrays";
    return false;
  }
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) { err = "cannot open " + path + " for writing"; return false; }
  const size_t nv = m.vertices.size() / 3, nt = m.triangles.size() / 3;
  std::fprintf(f, "ply\nformat ascii 1.0\n");
  if (!m.textureFile.empty()) std::fprintf(f, "comment TextureFile %s\n", m.textureFile.c_str());
  std::fprintf(f, "element vertex %zu\nproperty double x\nproperty double y\nproperty double z\n", nv);
  std::fprintf(f, "element face %zu\nproperty list uchar int vertex_indices\nproperty list uchar double texcoord\nend_header\n", nt);
  // %.17g: every double reads back to the same bits
  for (size_t v = 0; v < nv; v++)
    std::fprintf(f, "%.17g %.17g %.17g\n", m.vertices[3 * v], m.vertices[3 * v + 1], m.vertices[3 * v + 2]);
  for (size_t t = 0; t < nt; t++) {
    std::fprintf(f, "3 %d %d %d 6", m.triangles[3 * t], m.triangles[3 * t + 1], m.triangles[3 * t + 2]);
    for (int k = 0; k < 6; k++) std::fprintf(f, " %.17g", m.uv[6 * t + k]);
    std::fprintf(f, "\n");
  }
  const bool ok = std::ferror(f) == 0;
  if (std::fclose(f) != 0 || !ok) { err = "write failed: " + path; return false; }
  return true;
}

}  // namespace io
}  // namespace gdtp
