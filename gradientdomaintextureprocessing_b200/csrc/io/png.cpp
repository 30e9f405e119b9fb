// PNG codec for the texture I/O path (the reference links libpng:
// include/Misha/PNG.inl:10-120).  Decoding follows the PNG specification
// (chunks, zlib stream, per-row filters, Adam7) and then the reference's
// libpng transforms; encoding writes 8-bit RGB as PNGWriteColor does.
// zlib is loaded on first use, so libgdtp.so has no load-time dependency on it.
#include "io/texture_io.h"

#include <dlfcn.h>
#include <zlib.h>

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

namespace gdtp {
namespace io {
namespace {

struct Zlib {
  decltype(&::inflateInit_) f_inflateInit = nullptr;
  decltype(&::inflate) f_inflate = nullptr;
  decltype(&::inflateEnd) f_inflateEnd = nullptr;
  decltype(&::compressBound) f_compressBound = nullptr;
  decltype(&::compress2) f_compress2 = nullptr;
  bool ok = false;
};

const Zlib& zlib() {
  static Zlib z;
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = dlopen("libz.so.1", RTLD_NOW | RTLD_LOCAL);
    if (!h) return;
    z.f_inflateInit = reinterpret_cast<decltype(z.f_inflateInit)>(dlsym(h, "inflateInit_"));
    z.f_inflate = reinterpret_cast<decltype(z.f_inflate)>(dlsym(h, "inflate"));
    z.f_inflateEnd = reinterpret_cast<decltype(z.f_inflateEnd)>(dlsym(h, "inflateEnd"));
    z.f_compressBound = reinterpret_cast<decltype(z.f_compressBound)>(dlsym(h, "compressBound"));
    z.f_compress2 = reinterpret_cast<decltype(z.f_compress2)>(dlsym(h, "compress2"));
    z.ok = z.f_inflateInit && z.f_inflate && z.f_inflateEnd && z.f_compressBound && z.f_compress2;
  });
  return z;
}

// CRC-32 of the PNG specification (reflected polynomial 0xEDB88320, table driven)
uint32_t crc32_png(const unsigned char* p, size_t n) {
  static const std::array<uint32_t, 256> table = [] {
    std::array<uint32_t, 256> t{};
    for (uint32_t i = 0; i < 256; i++) {
      uint32_t c = i;
      for (int k = 0; k < 8; k++) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
      t[i] = c;
    }
    return t;
  }();
  uint32_t c = 0xFFFFFFFFu;
  for (size_t i = 0; i < n; i++) c = table[(c ^ p[i]) & 0xFF] ^ (c >> 8);
  return c ^ 0xFFFFFFFFu;
}

uint32_t rd32(const unsigned char* p) { return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | p[3]; }
void put32(std::vector<unsigned char>& o, uint32_t v) {
  for (int s = 24; s >= 0; s -= 8) o.push_back((unsigned char)(v >> s));
}

int channels_of(int colourType) {
  switch (colourType) {
    case 0: return 1;  // grey
    case 2: return 3;  // RGB
    case 3: return 1;  // palette index
    case 4: return 2;  // grey + alpha
    case 6: return 4;  // RGBA
    default: return 0;
  }
}

bool depth_allowed(int colourType, int depth) {
  switch (colourType) {
    case 0: return depth == 1 || depth == 2 || depth == 4 || depth == 8 || depth == 16;
    case 3: return depth == 1 || depth == 2 || depth == 4 || depth == 8;
    case 2: case 4: case 6: return depth == 8 || depth == 16;
    default: return false;
  }
}

// Adam7 passes: x start, y start, x step, y step; pass 0 alone when not interlaced
const int kAdam7[7][4] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4}, {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};

int paeth(int a, int b, int c) {
  const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
  if (pa <= pb && pa <= pc) return a;
  return pb <= pc ? b : c;
}

// undo the row filter of one row in place (prev: the previous row of the same pass, or zeros)
bool unfilter(int type, unsigned char* row, const unsigned char* prev, size_t n, size_t bpp) {
  switch (type) {
    case 0: return true;
    case 1: for (size_t i = bpp; i < n; i++) row[i] = (unsigned char)(row[i] + row[i - bpp]); return true;
    case 2: for (size_t i = 0; i < n; i++) row[i] = (unsigned char)(row[i] + prev[i]); return true;
    case 3:
      for (size_t i = 0; i < n; i++) row[i] = (unsigned char)(row[i] + ((int(i >= bpp ? row[i - bpp] : 0) + int(prev[i])) >> 1));
      return true;
    case 4:
      for (size_t i = 0; i < n; i++)
        row[i] = (unsigned char)(row[i] + paeth(i >= bpp ? row[i - bpp] : 0, prev[i], i >= bpp ? prev[i - bpp] : 0));
      return true;
    default: return false;
  }
}

}  // namespace

bool png_decode(const unsigned char* d, size_t n, Image8& img, bool headerOnly, std::string& err) {
  static const unsigned char kSig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  if (n < 8 || std::memcmp(d, kSig, 8) != 0) { err = "not a PNG file"; return false; }
  size_t pos = 8;
  uint32_t w = 0, h = 0;
  int depth = 0, ctype = -1, interlace = 0;
  bool seenHeader = false, seenEnd = false;
  std::vector<unsigned char> palette, zdata;
  while (pos + 12 <= n) {
    const uint32_t len = rd32(d + pos);
    if (len > n - pos - 12) { err = "truncated PNG chunk"; return false; }
    const unsigned char* type = d + pos + 4;
    const unsigned char* data = d + pos + 8;
    const bool critical = !(type[0] & 0x20);
    std::string tag;  // printable for messages: other bytes as \xNN
    for (int k = 0; k < 4; k++) {
      char hex[8];
      if (type[k] >= 32 && type[k] < 127) tag += char(type[k]);
      else std::snprintf(hex, sizeof(hex), "\\x%02X", type[k]), tag += hex;
    }
    if (crc32_png(type, size_t(len) + 4) != rd32(data + len)) {
      if (critical) { err = "CRC mismatch in PNG chunk " + tag; return false; }
      pos += 12 + size_t(len);
      continue;  // damaged ancillary chunk: ignored
    }
    if (!seenHeader && tag != "IHDR") { err = "PNG does not start with IHDR"; return false; }
    if (tag == "IHDR") {
      if (seenHeader || len != 13) { err = "bad PNG IHDR"; return false; }
      w = rd32(data), h = rd32(data + 4), depth = data[8], ctype = data[9], interlace = data[12];
      if (w == 0 || h == 0 || w > (1u << 24) || h > (1u << 24)) { err = "PNG size out of range"; return false; }
      if (!depth_allowed(ctype, depth) || data[10] != 0 || data[11] != 0 || interlace > 1) {
        err = "unsupported PNG format (colour type / bit depth / method)";
        return false;
      }
      if (uint64_t(w) * h > (uint64_t(1) << 30)) { err = "PNG larger than 2^30 pixels"; return false; }
      seenHeader = true;
      if (headerOnly) {
        img.width = int(w), img.height = int(h);
        img.rgb.clear();
        return true;
      }
    } else if (tag == "PLTE") {
      if (len == 0 || len % 3 != 0 || len > 768) { err = "bad PNG palette"; return false; }
      palette.assign(data, data + len);
    } else if (tag == "IDAT") {
      zdata.insert(zdata.end(), data, data + len);
    } else if (tag == "IEND") {
      seenEnd = true;
      break;
    } else if (critical) {
      err = "unknown critical PNG chunk " + tag;
      return false;
    }
    pos += 12 + size_t(len);
  }
  if (!seenHeader) { err = "PNG has no IHDR"; return false; }
  if (!seenEnd) { err = "PNG ends before IEND"; return false; }
  if (ctype == 3 && palette.empty()) { err = "palette PNG without PLTE"; return false; }

  const int ch = channels_of(ctype);
  const size_t bitsPP = size_t(ch) * depth, bpp = std::max<size_t>(1, bitsPP / 8);
  const int passes = interlace ? 7 : 1;
  size_t expected = 0;
  size_t pw[7] = {}, ph[7] = {};
  for (int p = 0; p < passes; p++) {
    const int xs = interlace ? kAdam7[p][0] : 0, ys = interlace ? kAdam7[p][1] : 0;
    const int dx = interlace ? kAdam7[p][2] : 1, dy = interlace ? kAdam7[p][3] : 1;
    pw[p] = w > uint32_t(xs) ? (w - xs + dx - 1) / dx : 0;
    ph[p] = h > uint32_t(ys) ? (h - ys + dy - 1) / dy : 0;
    if (pw[p] && ph[p]) expected += ph[p] * (1 + (pw[p] * bitsPP + 7) / 8);
  }

  const Zlib& z = zlib();
  if (!z.ok) { err = "zlib (libz.so.1) is not available"; return false; }
  std::vector<unsigned char> raw(expected);
  z_stream s;
  std::memset(&s, 0, sizeof(s));
  if (z.f_inflateInit(&s, ZLIB_VERSION, int(sizeof(z_stream))) != Z_OK) { err = "zlib inflateInit failed"; return false; }
  size_t inPos = 0, outPos = 0;
  int rc = Z_OK;
  while (outPos < expected) {
    const size_t inChunk = std::min<size_t>(zdata.size() - inPos, 1u << 30), outChunk = std::min<size_t>(expected - outPos, 1u << 30);
    s.next_in = zdata.data() + inPos;
    s.avail_in = uInt(inChunk);
    s.next_out = raw.data() + outPos;
    s.avail_out = uInt(outChunk);
    rc = z.f_inflate(&s, Z_NO_FLUSH);
    inPos += inChunk - s.avail_in;
    outPos += outChunk - s.avail_out;
    if (rc == Z_STREAM_END) break;
    if (rc != Z_OK || (inChunk - s.avail_in == 0 && outChunk - s.avail_out == 0)) break;
  }
  z.f_inflateEnd(&s);
  if (rc != Z_OK && rc != Z_STREAM_END) { err = "corrupt PNG image data (zlib)"; return false; }
  if (outPos < expected) { err = "PNG image data too short"; return false; }

  img.width = int(w), img.height = int(h);
  img.rgb.assign(size_t(w) * h * 3, 0);
  const size_t entries = palette.size() / 3;
  size_t off = 0;
  for (int p = 0; p < passes; p++) {
    if (!pw[p] || !ph[p]) continue;
    const int xs = interlace ? kAdam7[p][0] : 0, ys = interlace ? kAdam7[p][1] : 0;
    const int dx = interlace ? kAdam7[p][2] : 1, dy = interlace ? kAdam7[p][3] : 1;
    const size_t rowBytes = (pw[p] * bitsPP + 7) / 8;
    std::vector<unsigned char> zeros(rowBytes, 0);
    const unsigned char* prev = zeros.data();
    for (size_t y = 0; y < ph[p]; y++) {
      unsigned char* row = raw.data() + off + 1;
      if (!unfilter(raw[off], row, prev, rowBytes, bpp)) { err = "bad PNG filter type"; return false; }
      prev = row;
      off += 1 + rowBytes;
      unsigned char* dst = img.rgb.data() + 3 * ((ys + y * dy) * size_t(w));
      for (size_t x = 0; x < pw[p]; x++) {
        unsigned char* px = dst + 3 * (xs + x * dx);
        auto sample = [&](int k) -> int {
          if (depth == 8) return row[x * ch + k];
          if (depth == 16) return row[2 * (x * ch + k)];  // high byte
          const size_t bit = x * depth;                    // 1/2/4-bit: one channel
          return (row[bit >> 3] >> (8 - depth - int(bit & 7))) & ((1 << depth) - 1);
        };
        if (ctype == 3) {
          const int idx = sample(0);
          if (size_t(idx) >= entries) { err = "PNG palette index out of range"; return false; }
          std::memcpy(px, &palette[3 * idx], 3);
        } else if (ctype == 2 || ctype == 6) {
          for (int c = 0; c < 3; c++) px[c] = (unsigned char)sample(c);
        } else {  // grey, grey + alpha
          px[0] = px[1] = px[2] = (unsigned char)sample(0);
        }
      }
    }
  }
  return true;
}

bool png_encode_rgb(const Image8& img, std::vector<unsigned char>& out, std::string& err) {
  if (img.width <= 0 || img.height <= 0 || img.rgb.size() != size_t(img.width) * img.height * 3) {
    err = "bad image for PNG encoding";
    return false;
  }
  const Zlib& z = zlib();
  if (!z.ok) { err = "zlib (libz.so.1) is not available"; return false; }
  const size_t rowBytes = size_t(img.width) * 3, bpp = 3;
  std::vector<unsigned char> filtered(size_t(img.height) * (1 + rowBytes));
  std::vector<unsigned char> cand(rowBytes), best(rowBytes);
  std::vector<unsigned char> zeros(rowBytes, 0);
  for (int y = 0; y < img.height; y++) {
    const unsigned char* row = img.rgb.data() + size_t(y) * rowBytes;
    const unsigned char* prev = y ? row - rowBytes : zeros.data();
    // the filter with the smallest sum of |signed residual| (the usual adaptive choice)
    long long bestCost = -1;
    int bestType = 0;
    for (int t = 0; t < 5; t++) {
      long long cost = 0;
      for (size_t i = 0; i < rowBytes; i++) {
        const int a = i >= bpp ? row[i - bpp] : 0, b = prev[i], c = i >= bpp ? prev[i - bpp] : 0;
        const int pred = t == 0 ? 0 : t == 1 ? a : t == 2 ? b : t == 3 ? (a + b) >> 1 : paeth(a, b, c);
        cand[i] = (unsigned char)(row[i] - pred);
        cost += std::abs(int(static_cast<signed char>(cand[i])));
      }
      if (bestCost < 0 || cost < bestCost) bestCost = cost, bestType = t, best.swap(cand);
    }
    unsigned char* dst = filtered.data() + size_t(y) * (1 + rowBytes);
    dst[0] = (unsigned char)bestType;
    std::memcpy(dst + 1, best.data(), rowBytes);
  }
  uLongf zlen = z.f_compressBound(uLong(filtered.size()));
  std::vector<unsigned char> zbuf(zlen);
  if (z.f_compress2(zbuf.data(), &zlen, filtered.data(), uLong(filtered.size()), 6) != Z_OK) { err = "zlib compress failed"; return false; }
  out.clear();
  static const unsigned char kSig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  out.insert(out.end(), kSig, kSig + 8);
  auto chunk = [&](const char* tag, const unsigned char* data, size_t len) {
    put32(out, uint32_t(len));
    const size_t start = out.size();
    out.insert(out.end(), tag, tag + 4);
    if (len) out.insert(out.end(), data, data + len);
    put32(out, crc32_png(out.data() + start, len + 4));
  };
  unsigned char ihdr[13];
  for (int k = 0; k < 4; k++) ihdr[k] = (unsigned char)(uint32_t(img.width) >> (24 - 8 * k));
  for (int k = 0; k < 4; k++) ihdr[4 + k] = (unsigned char)(uint32_t(img.height) >> (24 - 8 * k));
  ihdr[8] = 8, ihdr[9] = 2, ihdr[10] = 0, ihdr[11] = 0, ihdr[12] = 0;
  chunk("IHDR", ihdr, 13);
  for (size_t o = 0; o < zlen; o += (1u << 20)) chunk("IDAT", zbuf.data() + o, std::min<size_t>(1u << 20, zlen - o));
  chunk("IEND", nullptr, 0);
  return true;
}

}  // namespace io
}  // namespace gdtp
