// Image targets: ImageLoader::load / ImageSaver::saveAsPNG
// (src/io/image_io.cpp:23-97).  The reference decodes with stb_image, resizes
// with stb_image_resize2 and writes with stb_image_write.  Here:
//   * decoding: PNG (8-bit, non-interlaced; grey, grey+alpha, RGB, RGBA,
//     palette) with a project-written DEFLATE decoder (RFC 1951) and the PNG
//     row filters (PNG specification, section 9), and binary PPM / PGM;
//   * aspect fit + pad on the GPU: scale = min((W - 2p) / w, (H - 2p) / h),
//     fit size = (int)(w * scale) x (int)(h * scale), centred on a black
//     canvas (the reference's geometry); the resampling is an area-weighted
//     box filter (downscale) / bilinear interpolation (upscale) in linear
//     8-bit values, not stb's Mitchell / Catmull-Rom kernels;
//   * writing: PNG with stored (uncompressed) DEFLATE blocks, bytes
//     (uint8)(clamp(v * 255, 0, 255)) like the reference.
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <cmath>
#include <fstream>
#include <string>
#include <vector>

#include "ds_common.cuh"
#include "ds_internal.h"

namespace {

// ---- DEFLATE (RFC 1951) ----------------------------------------------------
struct BitReader {
  const uint8_t* p;
  size_t n, pos = 0;
  uint32_t bitbuf = 0;
  int bitcnt = 0;
  bool bad = false;
  int bit() {
    if (bitcnt == 0) {
      if (pos >= n) {
        bad = true;
        return 0;
      }
      bitbuf = p[pos++];
      bitcnt = 8;
    }
    const int b = bitbuf & 1;
    bitbuf >>= 1;
    --bitcnt;
    return b;
  }
  uint32_t bits(int k) {  // LSB first
    uint32_t v = 0;
    for (int i = 0; i < k; ++i) v |= (uint32_t)bit() << i;
    return v;
  }
  void align() { bitcnt = 0; }
};

// Canonical Huffman decoding table: counts per length and symbols sorted by code.
struct Huffman {
  uint16_t count[16] = {0};
  uint16_t symbol[320] = {0};
  bool build(const uint8_t* lengths, int n) {
    memset(count, 0, sizeof(count));
    for (int i = 0; i < n; ++i) ++count[lengths[i]];
    count[0] = 0;
    int left = 1;
    for (int len = 1; len < 16; ++len) {
      left <<= 1;
      left -= count[len];
      if (left < 0) return false;  // over-subscribed
    }
    uint16_t offs[16];
    offs[1] = 0;
    for (int len = 1; len < 15; ++len) offs[len + 1] = offs[len] + count[len];
    for (int i = 0; i < n; ++i)
      if (lengths[i]) symbol[offs[lengths[i]]++] = (uint16_t)i;
    return true;
  }
  int decode(BitReader& br) const {
    int code = 0, first = 0, index = 0;
    for (int len = 1; len < 16; ++len) {
      code |= br.bit();
      const int c = count[len];
      if (code - c < first) return symbol[index + (code - first)];
      index += c;
      first += c;
      first <<= 1;
      code <<= 1;
      if (br.bad) return -1;
    }
    return -1;
  }
};

const uint16_t kLenBase[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                               31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
const uint8_t kLenExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                               2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
const uint16_t kDistBase[30] = {1,    2,    3,    4,    5,    7,     9,     13,    17,  25,
                                33,   49,   65,   97,   129,  193,   257,   385,   513, 769,
                                1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
const uint8_t kDistExtra[30] = {0, 0, 0, 0, 1, 1, 2, 2,  3,  3,  4,  4,  5,  5,  6,
                                6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};

// Output beyond `limit` bytes fails the decode: a small crafted stream could
// otherwise expand to gigabytes before the size check of its caller.
bool inflate_block(BitReader& br, const Huffman& lit, const Huffman& dist,
                   std::vector<uint8_t>& out, size_t limit) {
  for (;;) {
    int sym = lit.decode(br);
    if (sym < 0 || br.bad) return false;
    if (sym < 256) {
      if (out.size() >= limit) return false;
      out.push_back((uint8_t)sym);
    } else if (sym == 256) {
      return true;
    } else {
      sym -= 257;
      if (sym >= 29) return false;
      const int len = kLenBase[sym] + (int)br.bits(kLenExtra[sym]);
      const int ds = dist.decode(br);
      if (ds < 0 || ds >= 30) return false;
      const size_t d = kDistBase[ds] + br.bits(kDistExtra[ds]);
      if (d > out.size() || out.size() + (size_t)len > limit) return false;
      const size_t from = out.size() - d;
      for (int i = 0; i < len; ++i) out.push_back(out[from + i]);
    }
  }
}

bool inflate(const uint8_t* data, size_t n, std::vector<uint8_t>& out, size_t limit) {
  BitReader br{data, n};
  int last = 0;
  do {
    last = br.bit();
    const int type = (int)br.bits(2);
    if (type == 0) {  // stored
      br.align();
      if (br.pos + 4 > n) return false;
      const uint16_t len = (uint16_t)(data[br.pos] | (data[br.pos + 1] << 8));
      const uint16_t nlen = (uint16_t)(data[br.pos + 2] | (data[br.pos + 3] << 8));
      br.pos += 4;
      if ((uint16_t)~nlen != len || br.pos + len > n || out.size() + len > limit) return false;
      out.insert(out.end(), data + br.pos, data + br.pos + len);
      br.pos += len;
    } else if (type == 1) {  // fixed Huffman codes
      uint8_t l[288], d[30];
      for (int i = 0; i < 144; ++i) l[i] = 8;
      for (int i = 144; i < 256; ++i) l[i] = 9;
      for (int i = 256; i < 280; ++i) l[i] = 7;
      for (int i = 280; i < 288; ++i) l[i] = 8;
      for (int i = 0; i < 30; ++i) d[i] = 5;
      Huffman lit, dist;
      lit.build(l, 288);
      dist.build(d, 30);
      if (!inflate_block(br, lit, dist, out, limit)) return false;
    } else if (type == 2) {  // dynamic Huffman codes
      const int hlit = (int)br.bits(5) + 257, hdist = (int)br.bits(5) + 1;
      const int hclen = (int)br.bits(4) + 4;
      static const uint8_t order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5,
                                        11, 4,  12, 3, 13, 2, 14, 1, 15};
      uint8_t cl[19] = {0};
      for (int i = 0; i < hclen; ++i) cl[order[i]] = (uint8_t)br.bits(3);
      Huffman clh;
      if (!clh.build(cl, 19)) return false;
      uint8_t lens[320] = {0};
      int i = 0;
      while (i < hlit + hdist) {
        const int sym = clh.decode(br);
        if (sym < 0 || br.bad) return false;
        if (sym < 16) {
          lens[i++] = (uint8_t)sym;
        } else {
          int rep = 0;
          uint8_t val = 0;
          if (sym == 16) {
            if (i == 0) return false;
            val = lens[i - 1];
            rep = 3 + (int)br.bits(2);
          } else if (sym == 17) {
            rep = 3 + (int)br.bits(3);
          } else {
            rep = 11 + (int)br.bits(7);
          }
          if (i + rep > hlit + hdist) return false;
          while (rep--) lens[i++] = val;
        }
      }
      Huffman lit, dist;
      if (!lit.build(lens, hlit) || !dist.build(lens + hlit, hdist)) return false;
      if (!inflate_block(br, lit, dist, out, limit)) return false;
    } else {
      return false;
    }
    if (br.bad) return false;
  } while (!last);
  return true;
}

// ---- PNG ----------------------------------------------------------------------
uint32_t be32(const uint8_t* p) {
  return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}

uint32_t crc32_update(uint32_t crc, const uint8_t* p, size_t n) {
  static uint32_t table[256];
  static bool init = false;
  if (!init) {
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t c = i;
      for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
      table[i] = c;
    }
    init = true;
  }
  crc = ~crc;
  for (size_t i = 0; i < n; ++i) crc = table[(crc ^ p[i]) & 0xFF] ^ (crc >> 8);
  return ~crc;
}

int paeth(int a, int b, int c) {
  const int p = a + b - c, pa = abs(p - a), pb = abs(p - b), pc = abs(p - c);
  return (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
}

// Decodes to 8-bit RGB; false on anything unsupported or malformed.
bool decode_png(const std::vector<uint8_t>& f, int* w, int* h, std::vector<uint8_t>* rgb) {
  static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  if (f.size() < 8 || memcmp(f.data(), sig, 8) != 0) return false;
  size_t pos = 8;
  int W = 0, H = 0, depth = 0, ctype = 0, interlace = 0;
  std::vector<uint8_t> idat, palette;
  bool have_ihdr = false;
  while (pos + 12 <= f.size()) {
    const uint32_t len = be32(&f[pos]);
    if (pos + 12 + (size_t)len > f.size()) return false;
    const uint8_t* type = &f[pos + 4];
    const uint8_t* d = &f[pos + 8];
    if (!memcmp(type, "IHDR", 4) && len >= 13) {
      W = (int)be32(d);
      H = (int)be32(d + 4);
      depth = d[8];
      ctype = d[9];
      interlace = d[12];
      have_ihdr = true;
    } else if (!memcmp(type, "PLTE", 4)) {
      palette.assign(d, d + len);
    } else if (!memcmp(type, "IDAT", 4)) {
      idat.insert(idat.end(), d, d + len);
    } else if (!memcmp(type, "IEND", 4)) {
      break;
    }
    pos += 12 + len;
  }
  if (!have_ihdr || W <= 0 || H <= 0 || depth != 8 || interlace != 0) return false;
  if ((int64_t)W * H > (int64_t)1 << 28) return false;
  int ch = 0;
  switch (ctype) {
    case 0: ch = 1; break;
    case 2: ch = 3; break;
    case 3: ch = 1; break;
    case 4: ch = 2; break;
    case 6: ch = 4; break;
    default: return false;
  }
  if (ctype == 3 && palette.size() < 3) return false;
  if (idat.size() < 6) return false;
  std::vector<uint8_t> raw;
  raw.reserve((size_t)(W * ch + 1) * H);
  // zlib header / Adler-32 around the deflate stream; the filtered rows are
  // (stride + 1) * H bytes, more is malformed
  if (!inflate(idat.data() + 2, idat.size() - 6, raw, (size_t)(W * ch + 1) * H)) return false;
  const size_t stride = (size_t)W * ch;
  if (raw.size() < (stride + 1) * H) return false;
  std::vector<uint8_t> img(stride * H);
  for (int y = 0; y < H; ++y) {
    const uint8_t ft = raw[y * (stride + 1)];
    const uint8_t* src = &raw[y * (stride + 1) + 1];
    uint8_t* cur = &img[y * stride];
    const uint8_t* prev = y ? &img[(y - 1) * stride] : nullptr;
    for (size_t x = 0; x < stride; ++x) {
      const int a = x >= (size_t)ch ? cur[x - ch] : 0;
      const int b = prev ? prev[x] : 0;
      const int c = (prev && x >= (size_t)ch) ? prev[x - ch] : 0;
      int v = src[x];
      switch (ft) {
        case 0: break;
        case 1: v += a; break;
        case 2: v += b; break;
        case 3: v += (a + b) >> 1; break;
        case 4: v += paeth(a, b, c); break;
        default: return false;
      }
      cur[x] = (uint8_t)v;
    }
  }
  rgb->resize((size_t)W * H * 3);
  for (size_t i = 0; i < (size_t)W * H; ++i) {
    const uint8_t* s = &img[i * ch];
    uint8_t* o = &(*rgb)[i * 3];
    if (ctype == 3) {
      const size_t k = (size_t)s[0] * 3;
      if (k + 2 >= palette.size()) return false;
      o[0] = palette[k];
      o[1] = palette[k + 1];
      o[2] = palette[k + 2];
    } else if (ch <= 2) {
      o[0] = o[1] = o[2] = s[0];
    } else {
      o[0] = s[0];
      o[1] = s[1];
      o[2] = s[2];
    }
  }
  *w = W;
  *h = H;
  return true;
}

// Binary PPM (P6) / PGM (P5), maxval 255.
bool decode_pnm(const std::vector<uint8_t>& f, int* w, int* h, std::vector<uint8_t>* rgb) {
  if (f.size() < 3 || f[0] != 'P' || (f[1] != '6' && f[1] != '5')) return false;
  const int ch = f[1] == '6' ? 3 : 1;
  size_t pos = 2;
  int vals[3], nv = 0;
  while (nv < 3 && pos < f.size()) {
    while (pos < f.size() && (isspace(f[pos]) || f[pos] == '#')) {
      if (f[pos] == '#')
        while (pos < f.size() && f[pos] != '\n') ++pos;
      else
        ++pos;
    }
    int v = 0, digits = 0;
    while (pos < f.size() && isdigit(f[pos])) {
      v = v * 10 + (f[pos++] - '0');
      ++digits;
    }
    if (!digits) return false;
    vals[nv++] = v;
  }
  if (nv < 3 || vals[2] != 255 || vals[0] <= 0 || vals[1] <= 0) return false;
  ++pos;  // single whitespace
  const size_t n = (size_t)vals[0] * vals[1];
  if (pos + n * ch > f.size()) return false;
  rgb->resize(n * 3);
  for (size_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) (*rgb)[i * 3 + c] = f[pos + i * ch + (ch == 3 ? c : 0)];
  *w = vals[0];
  *h = vals[1];
  return true;
}

bool read_file(const char* path, std::vector<uint8_t>* out) {
  std::ifstream in(path, std::ios::binary);
  if (!in) return false;
  out->assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
  return true;
}

bool decode_any(const char* path, int* w, int* h, std::vector<uint8_t>* rgb) {
  std::vector<uint8_t> f;
  if (!path || !read_file(path, &f)) return false;
  return decode_png(f, w, h, rgb) || decode_pnm(f, w, h, rgb);
}

// ---- aspect fit + pad on the GPU --------------------------------------------
// Canvas pixel (x, y) inside the fitted rectangle samples the source: area
// average over the source footprint when shrinking (box filter), bilinear
// between source pixel centres when enlarging; values / 255; black outside.
__global__ void fit_kernel(const uint8_t* __restrict__ src, int sw, int sh, int fw, int fh, int ox,
                           int oy, int W, int H, float* __restrict__ dst) {
  const int64_t total = (int64_t)W * H;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % W), y = (int)(i / W);
    float r = 0.f, g = 0.f, b = 0.f;
    const int fx = x - ox, fy = y - oy;
    if (fx >= 0 && fx < fw && fy >= 0 && fy < fh) {
      const float sx = (float)sw / fw, sy = (float)sh / fh;
      if (sx > 1.f || sy > 1.f) {
        // box filter over [fx * sx, (fx + 1) * sx) x [fy * sy, (fy + 1) * sy)
        const float x0 = fx * sx, x1 = (fx + 1) * sx, y0 = fy * sy, y1 = (fy + 1) * sy;
        float wsum = 0.f;
        for (int v = (int)floorf(y0); v < (int)ceilf(y1) && v < sh; ++v) {
          const float wy = fminf(y1, v + 1.f) - fmaxf(y0, (float)v);
          for (int u = (int)floorf(x0); u < (int)ceilf(x1) && u < sw; ++u) {
            const float wx = fminf(x1, u + 1.f) - fmaxf(x0, (float)u);
            const float wgt = wx * wy;
            const uint8_t* p = src + ((size_t)v * sw + u) * 3;
            r += wgt * p[0];
            g += wgt * p[1];
            b += wgt * p[2];
            wsum += wgt;
          }
        }
        r /= wsum;
        g /= wsum;
        b /= wsum;
      } else {
        const float u = fminf(fmaxf((fx + 0.5f) * sx - 0.5f, 0.f), (float)(sw - 1));
        const float v = fminf(fmaxf((fy + 0.5f) * sy - 0.5f, 0.f), (float)(sh - 1));
        const int u0 = (int)u, v0 = (int)v;
        const int u1 = min(u0 + 1, sw - 1), v1 = min(v0 + 1, sh - 1);
        const float tu = u - u0, tv = v - v0;
        const uint8_t* p00 = src + ((size_t)v0 * sw + u0) * 3;
        const uint8_t* p01 = src + ((size_t)v0 * sw + u1) * 3;
        const uint8_t* p10 = src + ((size_t)v1 * sw + u0) * 3;
        const uint8_t* p11 = src + ((size_t)v1 * sw + u1) * 3;
        float c[3];
        for (int k = 0; k < 3; ++k) {
          const float top = p00[k] + (p01[k] - (float)p00[k]) * tu;
          const float bot = p10[k] + (p11[k] - (float)p10[k]) * tu;
          c[k] = top + (bot - top) * tv;
        }
        r = c[0];
        g = c[1];
        b = c[2];
      }
      r /= 255.f;
      g /= 255.f;
      b /= 255.f;
    }
    dst[i * 3 + 0] = r;
    dst[i * 3 + 1] = g;
    dst[i * 3 + 2] = b;
  }
}

void put32(std::vector<uint8_t>& v, uint32_t x) {
  v.push_back((uint8_t)(x >> 24));
  v.push_back((uint8_t)(x >> 16));
  v.push_back((uint8_t)(x >> 8));
  v.push_back((uint8_t)x);
}

void chunk(std::vector<uint8_t>& out, const char* type, const std::vector<uint8_t>& data) {
  put32(out, (uint32_t)data.size());
  const size_t start = out.size();
  out.insert(out.end(), type, type + 4);
  out.insert(out.end(), data.begin(), data.end());
  put32(out, crc32_update(0, &out[start], out.size() - start));
}

}  // namespace

extern "C" {

static int ds_image_probe_impl(const char* path, int* width, int* height) {
  if (!width || !height) return DS_ERR_ARG;
  std::vector<uint8_t> rgb;
  return decode_any(path, width, height, &rgb) ? DS_OK : DS_ERR_ARG;
}

static int ds_image_read_rgb8_impl(const char* path, uint8_t* rgb, int64_t capacity, int* width,
                       int* height) {
  if (!rgb || !width || !height) return DS_ERR_ARG;
  std::vector<uint8_t> img;
  int w = 0, h = 0;
  if (!decode_any(path, &w, &h, &img)) return DS_ERR_ARG;
  if ((int64_t)img.size() > capacity) return DS_ERR_ARG;
  memcpy(rgb, img.data(), img.size());
  *width = w;
  *height = h;
  return DS_OK;
}

int ds_image_fit(const uint8_t* src_rgb, int src_w, int src_h, int canvas_w, int canvas_h,
                 int padding, float* dst_rgb, int* fit_w, int* fit_h, ds_stream stream) {
  if (!src_rgb || !dst_rgb || src_w <= 0 || src_h <= 0 || canvas_w <= 0 || canvas_h <= 0 ||
      padding < 0 || 2 * padding >= canvas_w || 2 * padding >= canvas_h)
    return DS_ERR_ARG;
  const float scale = std::min((float)(canvas_w - 2 * padding) / src_w,
                               (float)(canvas_h - 2 * padding) / src_h);
  const int fw = std::max(1, (int)(src_w * scale)), fh = std::max(1, (int)(src_h * scale));
  const int ox = (canvas_w - fw) / 2, oy = (canvas_h - fh) / 2;
  const int64_t total = (int64_t)canvas_w * canvas_h;
  const unsigned blocks = (unsigned)std::min<int64_t>((total + 255) / 256, 148 * 16);
  fit_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(src_rgb, src_w, src_h, fw, fh, ox, oy,
                                                         canvas_w, canvas_h, dst_rgb);
  if (fit_w) *fit_w = fw;
  if (fit_h) *fit_h = fh;
  return ds::cuda_status(cudaGetLastError());
}

static int ds_image_write_png_impl(const char* path, const float* rgb, int width, int height) {
  if (!path || !rgb || width <= 0 || height <= 0) return DS_ERR_ARG;
  std::vector<uint8_t> raw;
  raw.reserve((size_t)(width * 3 + 1) * height);
  for (int y = 0; y < height; ++y) {
    raw.push_back(0);  // filter: none
    for (int x = 0; x < width * 3; ++x) {
      const float v = rgb[(size_t)y * width * 3 + x] * 255.f;
      raw.push_back((uint8_t)fminf(fmaxf(v, 0.f), 255.f));
    }
  }
  // zlib stream of stored blocks + Adler-32
  std::vector<uint8_t> z = {0x78, 0x01};
  for (size_t off = 0; off < raw.size() || off == 0; off += 65535) {
    const size_t len = std::min<size_t>(65535, raw.size() - off);
    const bool last = off + len >= raw.size();
    z.push_back(last ? 1 : 0);
    z.push_back((uint8_t)len);
    z.push_back((uint8_t)(len >> 8));
    z.push_back((uint8_t)~len);
    z.push_back((uint8_t)(~len >> 8));
    z.insert(z.end(), raw.begin() + off, raw.begin() + off + len);
    if (last) break;
  }
  uint32_t a = 1, b = 0;
  for (uint8_t c : raw) {
    a = (a + c) % 65521;
    b = (b + a) % 65521;
  }
  put32(z, (b << 16) | a);
  std::vector<uint8_t> png = {137, 80, 78, 71, 13, 10, 26, 10};
  std::vector<uint8_t> ihdr;
  put32(ihdr, (uint32_t)width);
  put32(ihdr, (uint32_t)height);
  ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});
  chunk(png, "IHDR", ihdr);
  chunk(png, "IDAT", z);
  chunk(png, "IEND", {});
  std::ofstream out(path, std::ios::binary);
  if (!out) return DS_ERR_ARG;
  out.write((const char*)png.data(), (std::streamsize)png.size());
  return out.good() ? DS_OK : DS_ERR_ARG;
}

// C++ exceptions (allocation, malformed numbers) become status codes at the ABI.
int ds_image_probe(const char* path, int* width, int* height) {
  try {
    return ds_image_probe_impl(path, width, height);
  } catch (const std::bad_alloc&) {
    return DS_ERR_OOM;
  } catch (...) {
    return DS_ERR_ARG;
  }
}

int ds_image_read_rgb8(const char* path, uint8_t* rgb, int64_t capacity, int* width, int* height) {
  try {
    return ds_image_read_rgb8_impl(path, rgb, capacity, width, height);
  } catch (const std::bad_alloc&) {
    return DS_ERR_OOM;
  } catch (...) {
    return DS_ERR_ARG;
  }
}

int ds_image_write_png(const char* path, const float* rgb, int width, int height) {
  try {
    return ds_image_write_png_impl(path, rgb, width, height);
  } catch (const std::bad_alloc&) {
    return DS_ERR_OOM;
  } catch (...) {
    return DS_ERR_ARG;
  }
}

}  // extern "C"
