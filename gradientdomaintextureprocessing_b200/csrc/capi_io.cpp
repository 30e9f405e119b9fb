// C ABI of the texture I/O path (host only; no device needed).
#include <cstring>
#include <string>
#include <vector>

#include "capi_internal.h"
#include "gdtp.h"
#include "io/texture_io.h"

using namespace gdtp;

extern "C" int gdtp_read_textured_mesh(const char* path, int64_t* nv, int64_t* nt, double* vertices, int32_t* triangles,
                                       double* uv) {
  return guarded("gdtp_read_textured_mesh", [&]() -> int {
    if (!path || !nv || !nt) return fail(GDTP_ERR_INVALID, "gdtp_read_textured_mesh: bad arguments");
    io::TexturedMesh m;
    std::string err;
    if (!io::read_ply_textured_mesh(path, m, err)) return fail(GDTP_ERR_INVALID, err);
    const int64_t v = int64_t(m.vertices.size() / 3), t = int64_t(m.triangles.size() / 3);
    if (vertices || triangles || uv) {
      if (!vertices || !triangles || !uv) return fail(GDTP_ERR_INVALID, "gdtp_read_textured_mesh: give all three outputs or none");
      if (*nv < v || *nt < t) return fail(GDTP_ERR_INVALID, "gdtp_read_textured_mesh: output arrays too small");
      std::memcpy(vertices, m.vertices.data(), m.vertices.size() * sizeof(double));
      for (size_t i = 0; i < m.triangles.size(); i++) triangles[i] = int32_t(m.triangles[i]);
      std::memcpy(uv, m.uv.data(), m.uv.size() * sizeof(double));
    }
    *nv = v, *nt = t;
    return GDTP_OK;
  });
}

extern "C" int gdtp_textured_mesh_texture_file(const char* path, char* name, int64_t* size) {
  return guarded("gdtp_textured_mesh_texture_file", [&]() -> int {
    if (!path || !size) return fail(GDTP_ERR_INVALID, "gdtp_textured_mesh_texture_file: bad arguments");
    io::TexturedMesh m;
    std::string err;
    if (!io::read_ply_textured_mesh(path, m, err)) return fail(GDTP_ERR_INVALID, err);
    if (name) {
      if (*size < int64_t(m.textureFile.size()) + 1) return fail(GDTP_ERR_INVALID, "gdtp_textured_mesh_texture_file: buffer too small");
      std::memcpy(name, m.textureFile.c_str(), m.textureFile.size() + 1);
    }
    *size = int64_t(m.textureFile.size()) + 1;
    return GDTP_OK;
  });
}

extern "C" int gdtp_write_textured_mesh(const char* path, const double* vertices, int64_t nv, const int32_t* triangles, int64_t nt,
                                        const double* uv, const char* texture_file) {
  return guarded("gdtp_write_textured_mesh", [&]() -> int {
    if (!path || nv < 0 || nt < 0 || nv > INT32_MAX || nt > INT32_MAX || (nv && !vertices) || (nt && (!triangles || !uv)))
      return fail(GDTP_ERR_INVALID, "gdtp_write_textured_mesh: bad arguments");
    io::TexturedMesh m;
    m.vertices.assign(vertices, vertices + nv * 3);
    m.triangles.assign(triangles, triangles + nt * 3);
    m.uv.assign(uv, uv + nt * 6);
    if (texture_file) m.textureFile = texture_file;
    std::string err;
    return io::write_ply_textured_mesh(path, m, err) ? GDTP_OK : fail(GDTP_ERR_INVALID, err);
  });
}

extern "C" int gdtp_read_image(const char* path, int* width, int* height, float* rgb) {
  return guarded("gdtp_read_image", [&]() -> int {
    if (!path || !width || !height) return fail(GDTP_ERR_INVALID, "gdtp_read_image: bad arguments");
    std::string err;
    int w = 0, h = 0;
    if (!rgb) {
      if (!io::read_image(path, nullptr, w, h, err)) return fail(GDTP_ERR_INVALID, err);
      *width = w, *height = h;
      return GDTP_OK;
    }
    std::vector<float> px;
    if (!io::read_image(path, &px, w, h, err)) return fail(GDTP_ERR_INVALID, err);
    if (*width != w || *height != h) return fail(GDTP_ERR_INVALID, "gdtp_read_image: width / height do not match the file");
    std::memcpy(rgb, px.data(), px.size() * sizeof(float));
    return GDTP_OK;
  });
}

extern "C" int gdtp_write_image(const char* path, const float* rgb, int width, int height) {
  return guarded("gdtp_write_image", [&]() -> int {
    if (!path || !rgb || width <= 0 || height <= 0) return fail(GDTP_ERR_INVALID, "gdtp_write_image: bad arguments");
    std::string err;
    return io::write_image(path, rgb, width, height, err) ? GDTP_OK : fail(GDTP_ERR_INVALID, err);
  });
}

extern "C" int gdtp_read_vector(const char* path, int64_t elem_bytes, int64_t* count, void* data) {
  return guarded("gdtp_read_vector", [&]() -> int {
    if (!path || !count || elem_bytes <= 0) return fail(GDTP_ERR_INVALID, "gdtp_read_vector: bad arguments");
    std::vector<unsigned char> buf;
    std::string err;
    if (!io::read_vector(path, size_t(elem_bytes), buf, err)) return fail(GDTP_ERR_INVALID, err);
    const int64_t n = int64_t(buf.size()) / elem_bytes;
    if (data) {
      if (*count < n) return fail(GDTP_ERR_INVALID, "gdtp_read_vector: output too small");
      std::memcpy(data, buf.data(), buf.size());
    }
    *count = n;
    return GDTP_OK;
  });
}

extern "C" int gdtp_write_vector(const char* path, int64_t elem_bytes, int64_t count, const void* data) {
  return guarded("gdtp_write_vector", [&]() -> int {
    if (!path || elem_bytes <= 0 || count < 0 || (count && !data)) return fail(GDTP_ERR_INVALID, "gdtp_write_vector: bad arguments");
    std::string err;
    return io::write_vector(path, size_t(elem_bytes), data, size_t(count), err) ? GDTP_OK : fail(GDTP_ERR_INVALID, err);
  });
}

static io::Padding padding_of(const int32_t* p) {
  io::Padding q;
  q.left = p[0], q.bottom = p[1], q.right = p[2], q.top = p[3];
  q.nonTrivial = q.left || q.bottom || q.right || q.top;
  return q;
}

extern "C" int gdtp_compute_padding(int width, int height, const double* uv, int64_t n_uv, int32_t* padding) {
  return guarded("gdtp_compute_padding", [&]() -> int {
    if (width <= 0 || height <= 0 || width > (1 << 24) || height > (1 << 24) || n_uv < 0 || (n_uv && !uv) || !padding) return fail(GDTP_ERR_INVALID, "gdtp_compute_padding: bad arguments");
    io::Padding p;
    std::string err;
    if (!io::compute_padding(width, height, uv, size_t(n_uv), p, err)) return fail(GDTP_ERR_INVALID, "gdtp_compute_padding: " + err);
    padding[0] = p.left, padding[1] = p.bottom, padding[2] = p.right, padding[3] = p.top;
    return GDTP_OK;
  });
}

extern "C" int gdtp_pad_texture_coordinates(const int32_t* padding, int width, int height, double* uv, int64_t n_uv, int unpad) {
  return guarded("gdtp_pad_texture_coordinates", [&]() -> int {
    if (!padding || width <= 0 || height <= 0 || width > (1 << 24) || height > (1 << 24) || n_uv < 0 || (n_uv && !uv)) return fail(GDTP_ERR_INVALID, "gdtp_pad_texture_coordinates: bad arguments");
    io::pad_texture_coordinates(padding_of(padding), width, height, uv, size_t(n_uv), unpad != 0);
    return GDTP_OK;
  });
}

extern "C" int gdtp_pad_image(const int32_t* padding, const float* in, int width, int height, float* out, int unpad) {
  return guarded("gdtp_pad_image", [&]() -> int {
    if (!padding || !in || !out) return fail(GDTP_ERR_INVALID, "gdtp_pad_image: bad arguments");
    std::vector<float> px;
    std::string err;
    if (!io::pad_image(padding_of(padding), in, width, height, px, unpad != 0, err)) return fail(GDTP_ERR_INVALID, err);
    std::memcpy(out, px.data(), px.size() * sizeof(float));
    return GDTP_OK;
  });
}
