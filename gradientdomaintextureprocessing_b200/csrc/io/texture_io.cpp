// Float RGB images, raw vectors and atlas padding of the texture I/O path
// (reference: include/Misha/Image.h:90-163, include/Src/VectorIO.h:9-58,
// include/Src/Padding.h:16-94).
#include "io/texture_io.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <strings.h>

namespace gdtp {
namespace io {
namespace {

// text after the last '.', compared case-insensitively as the reference's
// GetFileExtension + strcasecmp
std::string extension(const std::string& path) {
  const size_t dot = path.find_last_of('.');
  return dot == std::string::npos ? std::string() : path.substr(dot + 1);
}
bool is_ext(const std::string& path, const char* e) { return strcasecmp(extension(path).c_str(), e) == 0; }

bool read_file(const std::string& path, std::vector<unsigned char>& buf, std::string& err) {
  std::ifstream f(path, std::ios::binary);
  if (!f) { err = "cannot open " + path; return false; }
  buf.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  return true;
}
bool write_file(const std::string& path, const void* data, size_t n, std::string& err) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) { err = "cannot open " + path + " for writing"; return false; }
  const bool ok = std::fwrite(data, 1, n, f) == n;
  if (std::fclose(f) != 0 || !ok) { err = "write failed: " + path; return false; }
  return true;
}

// (unsigned char)min(255, max(0, (int)(v * 255 + 0.5))) in float arithmetic,
// product and sum rounded separately (Image.h:152-163)
unsigned char to_byte(float v) {
  volatile float t = v * 255.f;  // kept apart from the add: no fused multiply-add
  const float s = t + 0.5f;
  if (!(s > -2147483648.f && s < 2147483648.f)) return s > 0 ? 255 : 0;  // NaN and out of range
  return (unsigned char)std::min(255, std::max(0, int(s)));
}

}  // namespace

bool read_image(const std::string& path, std::vector<float>* rgb, int& width, int& height, std::string& err) {
  std::vector<unsigned char> buf;
  if (is_ext(path, "png")) {
    if (!read_file(path, buf, err)) return false;
    Image8 img;
    if (!png_decode(buf.data(), buf.size(), img, rgb == nullptr, err)) { err = path + ": " + err; return false; }
    width = img.width, height = img.height;
    if (rgb) {
      rgb->resize(img.rgb.size());
      for (size_t i = 0; i < img.rgb.size(); i++) (*rgb)[i] = float(img.rgb[i]) / 255.f;
    }
    return true;
  }
  if (is_ext(path, "normap")) {
    if (!read_file(path, buf, err)) return false;
    int32_t wh[2];
    if (buf.size() < 8) { err = path + ": truncated normap"; return false; }
    std::memcpy(wh, buf.data(), 8);
    if (wh[0] <= 0 || wh[1] <= 0 || size_t(wh[0]) > (buf.size() - 8) / 12 / size_t(wh[1])) {
      err = path + ": bad or truncated normap";
      return false;
    }
    width = wh[0], height = wh[1];
    if (rgb) {
      rgb->resize(size_t(width) * height * 3);
      std::memcpy(rgb->data(), buf.data() + 8, rgb->size() * sizeof(float));
    }
    return true;
  }
  err = path + ": unrecognised image extension (png or normap)";
  return false;
}

bool write_image(const std::string& path, const float* rgb, int width, int height, std::string& err) {
  if (!rgb || width <= 0 || height <= 0) { err = "bad image"; return false; }
  const size_t n = size_t(width) * height * 3;
  if (is_ext(path, "png")) {
    Image8 img;
    img.width = width, img.height = height;
    img.rgb.resize(n);
    for (size_t i = 0; i < n; i++) img.rgb[i] = to_byte(rgb[i]);
    std::vector<unsigned char> out;
    return png_encode_rgb(img, out, err) && write_file(path, out.data(), out.size(), err);
  }
  if (is_ext(path, "normap")) {
    std::vector<unsigned char> out(8 + n * sizeof(float));
    const int32_t wh[2] = {width, height};
    std::memcpy(out.data(), wh, 8);
    std::memcpy(out.data() + 8, rgb, n * sizeof(float));
    return write_file(path, out.data(), out.size(), err);
  }
  err = path + ": unrecognised image extension (png or normap)";
  return false;
}

bool read_vector(const std::string& path, size_t elemBytes, std::vector<unsigned char>& data, std::string& err) {
  std::vector<unsigned char> buf;
  if (elemBytes == 0) { err = "element size 0"; return false; }
  if (!read_file(path, buf, err)) return false;
  int32_t n = 0;
  if (buf.size() < 4) { err = path + ": truncated vector file"; return false; }
  std::memcpy(&n, buf.data(), 4);
  if (n < 0 || size_t(n) > (buf.size() - 4) / elemBytes) { err = path + ": vector file shorter than its count"; return false; }
  data.assign(buf.begin() + 4, buf.begin() + 4 + size_t(n) * elemBytes);
  return true;
}

bool write_vector(const std::string& path, size_t elemBytes, const void* data, size_t count, std::string& err) {
  if (count > size_t(INT32_MAX)) { err = "vector too long for an int32 count"; return false; }
  if (elemBytes == 0 || (count && elemBytes > (SIZE_MAX - 4) / count)) { err = "bad element size"; return false; }
  std::vector<unsigned char> out(4 + count * elemBytes);
  const int32_t n = int32_t(count);
  std::memcpy(out.data(), &n, 4);
  if (count) std::memcpy(out.data() + 4, data, count * elemBytes);
  return write_file(path, out.data(), out.size(), err);
}

// Padding.h:16-46: the texel grid must hold every texture coordinate at least
// half a texel inside; the padded size is then rounded up to multiples of 8 by
// growing left / bottom
bool compute_padding(int width, int height, const double* uv, size_t nUv, Padding& p, std::string& err) {
  p = Padding();
  if (nUv == 0) return true;
  for (size_t i = 0; i < 2 * nUv; i++)
    if (!(std::fabs(uv[i]) <= 1e6)) { err = "texture coordinate not finite or beyond 1e6"; return false; }
  const double pixMin[2] = {0.5 / double(width), 0.5 / double(height)};
  const double pixMax[2] = {(double(width) - 0.5) / double(width), (double(height) - 0.5) / double(height)};
  double tMin[2] = {uv[0], uv[1]}, tMax[2] = {uv[0], uv[1]};
  for (size_t i = 0; i < nUv; i++)
    for (int c = 0; c < 2; c++) tMin[c] = std::min(tMin[c], uv[2 * i + c]), tMax[c] = std::max(tMax[c], uv[2 * i + c]);
  const double pad[4] = {tMin[0] < pixMin[0] ? std::ceil((pixMin[0] - tMin[0]) * double(width)) : 0.0,
                         tMin[1] < pixMin[1] ? std::ceil((pixMin[1] - tMin[1]) * double(height)) : 0.0,
                         tMax[0] > pixMax[0] ? std::ceil((tMax[0] - pixMax[0]) * double(width)) : 0.0,
                         tMax[1] > pixMax[1] ? std::ceil((tMax[1] - pixMax[1]) * double(height)) : 0.0};
  for (double d : pad)
    if (d > 16777216.0) { err = "padding beyond 2^24 texels"; return false; }
  p.left = int(pad[0]), p.bottom = int(pad[1]), p.right = int(pad[2]), p.top = int(pad[3]);
  const int newW = width + p.left + p.right, newH = height + p.bottom + p.top;
  p.left += 8 * ((newW - 1) / 8 + 1) - newW;
  p.bottom += 8 * ((newH - 1) / 8 + 1) - newH;
  p.nonTrivial = p.left || p.right || p.bottom || p.top;
  return true;
}

// Padding.h:76-94.  The loop-invariant divisions are multiplies by the
// reciprocal, as the reference's release build computes them (its Makefile
// builds with -ffast-math, whose reciprocal-math rewrites x / c as
// x * (1 / c)); the plain quotient differs in the last bit for ~10-20 % of
// coordinates.
void pad_texture_coordinates(const Padding& p, int width, int height, double* uv, size_t nUv, bool unpad) {
  const double newW = double(width) + p.left + p.right, newH = double(height) + p.bottom + p.top;
  const double rx = unpad ? 1.0 / double(width) : 1.0 / newW, ry = unpad ? 1.0 / double(height) : 1.0 / newH;
  for (size_t i = 0; i < nUv; i++) {
    double& u = uv[2 * i];
    double& v = uv[2 * i + 1];
    if (!unpad) {
      u = (u * double(width) + double(p.left)) * rx;
      v = (v * double(height) + double(p.bottom)) * ry;
    } else {
      u = (u * newW - double(p.left)) * rx;
      v = (v * newH - double(p.bottom)) * ry;
    }
  }
}

// Padding.h:48-74: PaddImage repeats the edge texels, UnpaddImage crops
bool pad_image(const Padding& p, const float* in, int width, int height, std::vector<float>& out, bool unpad, std::string& err) {
  if (!in || width <= 0 || height <= 0 || p.left < 0 || p.right < 0 || p.bottom < 0 || p.top < 0) { err = "bad image or padding"; return false; }
  if (!unpad) {
    const long long wl = (long long)width + p.left + p.right, hl = (long long)height + p.bottom + p.top;
    if (wl > (1 << 24) || hl > (1 << 24)) { err = "padded image larger than 2^24 texels on a side"; return false; }
    const int w = int(wl), h = int(hl);
    out.resize(size_t(w) * h * 3);
    for (int j = 0; j < h; j++) {
      const int sj = std::min(std::max(0, j - p.bottom), height - 1);
      for (int i = 0; i < w; i++) {
        const int si = std::min(std::max(0, i - p.left), width - 1);
        std::memcpy(&out[3 * (size_t(j) * w + i)], &in[3 * (size_t(sj) * width + si)], 3 * sizeof(float));
      }
    }
    return true;
  }
  const long long wl = (long long)width - p.left - p.right, hl = (long long)height - p.bottom - p.top;
  if (wl <= 0 || hl <= 0) { err = "padding larger than the image"; return false; }
  const int w = int(wl), h = int(hl);
  out.resize(size_t(w) * h * 3);
  for (int j = 0; j < h; j++)
    std::memcpy(&out[3 * size_t(j) * w], &in[3 * (size_t(p.bottom + j) * width + p.left)], 3 * size_t(w) * sizeof(float));
  return true;
}

}  // namespace io
}  // namespace gdtp
