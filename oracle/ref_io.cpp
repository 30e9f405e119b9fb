// Oracle for the texture I/O path: runs the UNMODIFIED reference readers and
// padding helpers (compiled from the reference's own headers, never copied) on a
// given file and dumps what they produce, in the "GDTPDMP1" named-array format
// that oracle/gdd.py reads.  Test infrastructure only: nothing in the product
// links or runs this program.
//
//   gdtp_ref_io ply <mesh.ply> <out.gdd>
//       ReadTexturedMesh (include/Src/SimpleMesh.h:118-160) without a texture:
//       "vertices" (nv x 3), "triangles" (nt x 3), "uv" (3 nt x 2)
//   gdtp_ref_io vf <field.vf> <out.gdd>
//       ReadVector<Point2D<double>> (include/Src/VectorIO.h:9-20): "field" (n x 2)
//   gdtp_ref_io pad <width> <height> <uv.f64> <out.gdd>
//       ComputePadding (include/Src/Padding.h:16-46) on raw float64 (u, v) pairs,
//       then PaddTextureCoordinates / UnpaddTextureCoordinates (:76-94):
//       "padding" {left, bottom, right, top, nonTrivial}, "padded", "unpadded"
//   gdtp_ref_io writemesh <mesh.ply> <out.ply>
//       ReadTexturedMesh then WriteTexturedMesh (SimpleMesh.h:93-116) with an
//       atlas comment, so the tests can read a file the reference wrote
#define PNG_INCLUDED 1
void PNGWriteColor(const char*, const unsigned char*, int, int) {}
unsigned char* PNGReadColor(const char*, int&, int&) { return nullptr; }

#include <Src/SimpleMesh.h>
#include <Src/VectorIO.h>
#include <Src/Padding.h>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace {

struct Dump {
  FILE* f = nullptr;
  explicit Dump(const char* path) {
    f = fopen(path, "wb");
    if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
    fwrite("GDTPDMP1", 1, 8, f);
  }
  ~Dump() { if (f) fclose(f); }
  void put(const std::string& name, int code, int64_t rows, int64_t cols, const void* data, size_t bytes) {
    uint32_t n = (uint32_t)name.size();
    fwrite(&n, 4, 1, f);
    fwrite(name.data(), 1, n, f);
    uint8_t c = (uint8_t)code;
    fwrite(&c, 1, 1, f);
    uint32_t nd = 2;
    fwrite(&nd, 4, 1, f);
    int64_t dims[2] = {rows, cols};
    fwrite(dims, 8, 2, f);
    if (bytes) fwrite(data, 1, bytes, f);
  }
};

int ply(const char* in, const char* out) {
  TexturedMesh mesh;
  if (!ReadTexturedMesh(mesh, in, NULL)) { fprintf(stderr, "ReadTexturedMesh failed: %s\n", in); return 3; }
  std::vector<double> v, uv;
  std::vector<int> t;
  for (const auto& p : mesh.vertices) for (int c = 0; c < 3; c++) v.push_back(p[c]);
  for (const auto& tri : mesh.triangles) for (int c = 0; c < 3; c++) t.push_back(tri[c]);
  for (const auto& q : mesh.textureCoordinates) for (int c = 0; c < 2; c++) uv.push_back(q[c]);
  Dump d(out);
  d.put("vertices", 2, (int64_t)mesh.vertices.size(), 3, v.data(), v.size() * 8);
  d.put("triangles", 1, (int64_t)mesh.triangles.size(), 3, t.data(), t.size() * 4);
  d.put("uv", 2, (int64_t)mesh.textureCoordinates.size(), 2, uv.data(), uv.size() * 8);
  return 0;
}

int vf(const char* in, const char* out) {
  std::vector<Point2D<double>> field;
  if (!ReadVector(field, in)) return 3;
  std::vector<double> f;
  for (const auto& p : field) for (int c = 0; c < 2; c++) f.push_back(p[c]);
  Dump d(out);
  d.put("field", 2, (int64_t)field.size(), 2, f.data(), f.size() * 8);
  return 0;
}

int pad(int width, int height, const char* in, const char* out) {
  FILE* fi = fopen(in, "rb");
  if (!fi) return 3;
  std::vector<double> raw;
  double buf[2];
  while (fread(buf, 8, 2, fi) == 2) raw.push_back(buf[0]), raw.push_back(buf[1]);
  fclose(fi);
  std::vector<Point2D<double>> uv(raw.size() / 2);
  for (size_t i = 0; i < uv.size(); i++) uv[i] = Point2D<double>(raw[2 * i], raw[2 * i + 1]);
  Padding p;
  ComputePadding(p, width, height, uv);
  std::vector<Point2D<double>> padded = uv;
  PaddTextureCoordinates(p, width, height, padded);
  std::vector<Point2D<double>> unpadded = padded;
  UnpaddTextureCoordinates(p, width, height, unpadded);
  int pv[5] = {p.left, p.bottom, p.right, p.top, p.nonTrivial ? 1 : 0};
  std::vector<double> a, b;
  for (const auto& q : padded) a.push_back(q[0]), a.push_back(q[1]);
  for (const auto& q : unpadded) b.push_back(q[0]), b.push_back(q[1]);
  Dump d(out);
  d.put("padding", 1, 5, 1, pv, sizeof(pv));
  d.put("padded", 2, (int64_t)padded.size(), 2, a.data(), a.size() * 8);
  d.put("unpadded", 2, (int64_t)unpadded.size(), 2, b.data(), b.size() * 8);
  return 0;
}

int writemesh(const char* in, const char* out) {
  TexturedMesh mesh;
  if (!ReadTexturedMesh(mesh, in, NULL)) return 3;
  WriteTexturedMesh(mesh, out, "atlas.png");
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  const std::string mode = argc > 1 ? argv[1] : "";
  if (mode == "ply" && argc == 4) return ply(argv[2], argv[3]);
  if (mode == "vf" && argc == 4) return vf(argv[2], argv[3]);
  if (mode == "pad" && argc == 6) return pad(atoi(argv[2]), atoi(argv[3]), argv[4], argv[5]);
  if (mode == "writemesh" && argc == 4) return writemesh(argv[2], argv[3]);
  fprintf(stderr, "usage: %s ply|vf <in> <out.gdd> | pad <w> <h> <uv.f64> <out.gdd> | writemesh <in.ply> <out.ply>\n", argv[0]);
  return 1;
}
