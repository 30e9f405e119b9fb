// Host-side texture I/O of the texel-FEM apps: textured meshes (PLY), colour
// and normal textures (8-bit PNG, raw float "normap"), raw vectors (".vf"
// tangent fields), and the atlas padding that the apps apply before building
// the texel grid.  Behaviour follows the reference's readers and writers
// (file:line in fabianprada/GradientDomainTextureProcessing):
//   ReadTexturedMesh / WriteTexturedMesh   include/Src/SimpleMesh.h:93-160
//     over the PLY reader of include/Misha/PlyFile.inl (ASCII items through
//     atof / atoi, binary items in their declared type, byte-swapped when the
//     file's endianness differs)
//   Image<Point3D<float>>::read / write     include/Misha/Image.h:90-163
//     over PNGReadColor / PNGWriteColor     include/Misha/PNG.inl:10-120
//   ReadVector / WriteVector / ReadBinaryImage / WriteBinaryImage
//                                           include/Src/VectorIO.h:9-58
//   ComputePadding, Padd/Unpadd Image and TextureCoordinates
//                                           include/Src/Padding.h:16-94
// Images are row-major RGB with row 0 first (the first PNG row), pixel (i, j)
// at index 3 (j width + i), as the reference's Image<>.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace gdtp {
namespace io {

struct TexturedMesh {
  std::vector<double> vertices;  // nv x 3
  std::vector<int> triangles;    // nt x 3
  std::vector<double> uv;        // nt x 3 x 2, per corner
  std::string textureFile;       // from a "comment TextureFile <name>" header line, if any
};

// A PLY file with a "vertex" element (x, y, z) and a "face" element
// (vertex_indices list, texcoord list of 2 values per corner).  Faces with
// more than three corners keep their first three, as the reference does.
bool read_ply_textured_mesh(const std::string& path, TexturedMesh& m, std::string& err);
// ASCII PLY with full double precision, the reference writer's layout
bool write_ply_textured_mesh(const std::string& path, const TexturedMesh& m, std::string& err);

// 8-bit RGB image, row 0 first
struct Image8 {
  int width = 0, height = 0;
  std::vector<unsigned char> rgb;
};
// PNG of any standard colour type, bit depth and interlacing, reduced to 8-bit
// RGB with the reference's transforms: 16-bit samples keep their high byte,
// 1/2/4-bit samples are unpacked without rescaling, palette indices are looked
// up, alpha is dropped, grey is copied to all three channels.  headerOnly: the
// size only.
bool png_decode(const unsigned char* data, size_t size, Image8& img, bool headerOnly, std::string& err);
// 8-bit RGB, not interlaced, per-row adaptive filter, zlib level 6
bool png_encode_rgb(const Image8& img, std::vector<unsigned char>& out, std::string& err);

// Float RGB images by file extension: "png" (8-bit, value / 255) or "normap"
// (int32 width, int32 height, width x height float triples).  rgb == nullptr
// reads the size only.
bool read_image(const std::string& path, std::vector<float>* rgb, int& width, int& height, std::string& err);
// "png": each value v becomes min(255, max(0, (int)(v * 255 + 0.5))) in float
// arithmetic; "normap": raw floats
bool write_image(const std::string& path, const float* rgb, int width, int height, std::string& err);

// int32 count, then count elements of elemBytes each
bool read_vector(const std::string& path, size_t elemBytes, std::vector<unsigned char>& data, std::string& err);
bool write_vector(const std::string& path, size_t elemBytes, const void* data, size_t count, std::string& err);

struct Padding {
  int left = 0, bottom = 0, right = 0, top = 0;
  bool nonTrivial = false;
};
// false (with err) for texture coordinates that are not finite or beyond 1e6
bool compute_padding(int width, int height, const double* uv, size_t nUv, Padding& p, std::string& err);
// uv: nUv (u, v) pairs in place; unpad reverses
void pad_texture_coordinates(const Padding& p, int width, int height, double* uv, size_t nUv, bool unpad);
// pad: out is (width + left + right) x (height + bottom + top), edge texels
// repeated; unpad: out is (width - left - right) x (height - bottom - top)
bool pad_image(const Padding& p, const float* in, int width, int height, std::vector<float>& out, bool unpad, std::string& err);

}  // namespace io
}  // namespace gdtp
