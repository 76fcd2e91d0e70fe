// mrc.cpp -- MRC reader/writer and text inputs of the `tilt` drop-in.
// Byte layout and rules: crates/imod-mrc/src/{header,read,write}.rs,
// crates/imod-transforms/src/tilt.rs, apps/tilt/src/main.rs:232-326.
#include "mrc.h"

#include <math.h>
#include <string.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace mrc {

namespace {
struct Out {
  uint8_t *p;
  bool be;
  size_t o = 0;
  void raw(const void *d, size_t n) { memcpy(p + o, d, n); o += n; }
  template <class T> void put(T v) {
    uint8_t b[sizeof(T)];
    memcpy(b, &v, sizeof(T));
    if (be) std::reverse(b, b + sizeof(T));
    raw(b, sizeof(T));
  }
};
struct In {
  const uint8_t *p;
  bool be;
  size_t o = 0;
  void raw(void *d, size_t n) { memcpy(d, p + o, n); o += n; }
  template <class T> T get() {
    uint8_t b[sizeof(T)];
    raw(b, sizeof(T));
    if (be) std::reverse(b, b + sizeof(T));
    T v;
    memcpy(&v, b, sizeof(T));
    return v;
  }
};
}  // namespace

Header Header::make(int32_t nx, int32_t ny, int32_t nz, int32_t mode) {
  Header h;
  h.nx = nx; h.ny = ny; h.nz = nz; h.mode = mode;
  h.mx = nx; h.my = ny; h.mz = nz;
  h.xlen = (float)nx; h.ylen = (float)ny; h.zlen = (float)nz;
  h.imod_stamp = IMOD_STAMP;
  return h;
}

bool Header::add_label(const std::string &text) {
  if (nlabl < 0 || nlabl >= 10) return false;
  size_t n = std::min<size_t>(text.size(), 80);
  memcpy(labels[nlabl], text.data(), n);
  for (size_t i = n; i < 80; ++i) labels[nlabl][i] = ' ';
  ++nlabl;
  return true;
}

std::string Header::label(int idx) const {
  if (idx < 0 || idx >= nlabl || idx >= 10) return std::string();
  int end = 80;
  while (end > 0 && (labels[idx][end - 1] == ' ' || labels[idx][end - 1] == 0)) --end;
  return std::string(labels[idx], end);
}

bool Header::is_old_style() const { return nversion == 0 && memcmp(cmap, "MAP ", 4) != 0; }

int Header::bytes_per_pixel() const {
  switch (mode) {
    case BYTE: return 1;
    case SHORT: return 2;
    case FLOAT: return 4;
    case COMPLEX_SHORT: return 4;
    case COMPLEX_FLOAT: return 8;
    case USHORT: return 2;
    case HALF: return 2;
    case RGB: return 3;
    case FOURBIT: return 1;
    default: return 1;  // unknown modes are sized as bytes (slice_size_bytes)
  }
}

size_t Header::slice_bytes() const {
  if (mode == FOURBIT) return (size_t)(nx + 1) / 2 * ny;
  return (size_t)nx * ny * bytes_per_pixel();
}

void Header::to_bytes(uint8_t out[1024], bool be) const {
  Out w{out, be};
  w.put(nx); w.put(ny); w.put(nz); w.put(mode);
  w.put(nxstart); w.put(nystart); w.put(nzstart);
  w.put(mx); w.put(my); w.put(mz);
  w.put(xlen); w.put(ylen); w.put(zlen);
  w.put(alpha); w.put(beta); w.put(gamma);
  w.put(mapc); w.put(mapr); w.put(maps);
  w.put(amin); w.put(amax); w.put(amean);
  w.put(ispg); w.put(next);
  w.put(creatid); w.raw(blank, 6);
  w.raw(ext_type, 4);
  w.put(nversion);
  w.raw(blank2, 16);
  w.put(nint); w.put(nreal); w.put(sub); w.put(zfac);
  w.put(min2); w.put(max2); w.put(min3); w.put(max3);
  w.put(imod_stamp); w.put(imod_flags);
  w.put(idtype); w.put(lens); w.put(nd1); w.put(nd2); w.put(vd1); w.put(vd2);
  for (float t : tilt_angles) w.put(t);
  w.put(xorg); w.put(yorg); w.put(zorg);
  w.raw(cmap, 4); w.raw(stamp, 4);
  w.put(rms);
  w.put(nlabl);
  w.raw(labels, 800);
}

Header Header::from_bytes(const uint8_t in[1024], bool be) {
  In r{in, be};
  Header h;
  h.nx = r.get<int32_t>(); h.ny = r.get<int32_t>(); h.nz = r.get<int32_t>(); h.mode = r.get<int32_t>();
  h.nxstart = r.get<int32_t>(); h.nystart = r.get<int32_t>(); h.nzstart = r.get<int32_t>();
  h.mx = r.get<int32_t>(); h.my = r.get<int32_t>(); h.mz = r.get<int32_t>();
  h.xlen = r.get<float>(); h.ylen = r.get<float>(); h.zlen = r.get<float>();
  h.alpha = r.get<float>(); h.beta = r.get<float>(); h.gamma = r.get<float>();
  h.mapc = r.get<int32_t>(); h.mapr = r.get<int32_t>(); h.maps = r.get<int32_t>();
  h.amin = r.get<float>(); h.amax = r.get<float>(); h.amean = r.get<float>();
  h.ispg = r.get<int32_t>(); h.next = r.get<int32_t>();
  h.creatid = r.get<int16_t>(); r.raw(h.blank, 6);
  r.raw(h.ext_type, 4);
  h.nversion = r.get<int32_t>();
  r.raw(h.blank2, 16);
  h.nint = r.get<int16_t>(); h.nreal = r.get<int16_t>(); h.sub = r.get<int16_t>(); h.zfac = r.get<int16_t>();
  h.min2 = r.get<float>(); h.max2 = r.get<float>(); h.min3 = r.get<float>(); h.max3 = r.get<float>();
  h.imod_stamp = r.get<int32_t>(); h.imod_flags = r.get<int32_t>();
  h.idtype = r.get<int16_t>(); h.lens = r.get<int16_t>(); h.nd1 = r.get<int16_t>(); h.nd2 = r.get<int16_t>();
  h.vd1 = r.get<int16_t>(); h.vd2 = r.get<int16_t>();
  for (float &t : h.tilt_angles) t = r.get<float>();
  h.xorg = r.get<float>(); h.yorg = r.get<float>(); h.zorg = r.get<float>();
  r.raw(h.cmap, 4); r.raw(h.stamp, 4);
  h.rms = r.get<float>();
  h.nlabl = r.get<int32_t>();
  r.raw(h.labels, 800);
  return h;
}

static bool dims_reasonable(const Header &h) {
  return h.nx > 0 && h.ny > 0 && h.nz > 0 && h.nx < 100000 && h.ny < 100000 && h.nz < 1000000;
}

// IEEE 754 binary32 -> binary16, round to nearest, ties to even (the inverse of
// f16_to_f32 below on every half value).  Mode-12 output: the reference reads
// it (read.rs:468-499) but has no writer for it.
uint16_t f32_to_f16(float f) {
  uint32_t x;
  memcpy(&x, &f, 4);
  const uint32_t sign = (x >> 16) & 0x8000u, ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u)  // infinity, or NaN (quiet, upper payload bits kept)
    return (uint16_t)(sign | 0x7c00u | (ax > 0x7f800000u ? 0x200u | ((ax >> 13) & 0x3ffu) : 0u));
  if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);  // >= 65520 rounds to infinity
  if (ax < 0x38800000u) {  // below 2^-14: a subnormal half (or zero)
    const int e = (int)(ax >> 23);
    if (e < 102) return (uint16_t)sign;  // below 2^-25
    const uint32_t m = (ax & 0x7fffffu) | 0x800000u;  // value = m * 2^(e-150), unit 2^-24
    const int shift = 126 - e;                         // 14..24
    uint32_t r = m >> shift;
    const uint32_t rem = m & ((1u << shift) - 1u), half = 1u << (shift - 1);
    if (rem > half || (rem == half && (r & 1u))) ++r;  // may carry into the smallest normal
    return (uint16_t)(sign | r);
  }
  uint32_t r = ((((ax >> 23) - 127u + 15u) << 10) | ((ax & 0x7fffffu) >> 13));
  const uint32_t rem = ax & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (r & 1u))) ++r;  // a carry moves into the exponent
  return (uint16_t)(sign | r);
}

float f16_to_f32(uint16_t bits) {  // crates/imod-mrc/src/read.rs:468-499
  uint32_t sign = (bits >> 15) & 1, exponent = (bits >> 10) & 0x1F, mant = bits & 0x3FF, out;
  if (exponent == 0) {
    if (mant == 0) {
      out = sign << 31;
    } else {
      uint32_t m = mant;
      int e = 0;
      while ((m & 0x400) == 0) { m <<= 1; ++e; }
      uint32_t exp = (uint32_t)(127 - 15 + 1 - e);
      out = (sign << 31) | (exp << 23) | ((m & 0x3FF) << 13);
    }
  } else if (exponent == 31) {
    out = (sign << 31) | (0xFFu << 23) | (mant << 13);
  } else {
    out = (sign << 31) | ((exponent - 15 + 127) << 23) | (mant << 13);
  }
  float f;
  memcpy(&f, &out, 4);
  return f;
}

bool Reader::open(const std::string &path, std::string *err) {
  f_ = fopen(path.c_str(), "rb");
  if (!f_) { if (err) *err = "No such file or directory (os error 2)"; return false; }
  uint8_t b[1024];
  if (fread(b, 1, 1024, f_) != 1024) { if (err) *err = "Invalid MRC header: failed to fill whole buffer"; return false; }
  Header h = Header::from_bytes(b, false);
  swapped_ = h.is_swapped() || !dims_reasonable(h);
  if (swapped_) {
    h = Header::from_bytes(b, true);
    if (!dims_reasonable(h)) {
      if (err) *err = "Invalid MRC header: unreasonable dimensions even after byte-swap";
      return false;
    }
  }
  if (h.is_old_style()) {  // read.rs:54-83: origin fields shifted in pre-2014 headers
    float ox = h.yorg, oy = h.zorg, oz = h.xorg;
    h.xorg = ox; h.yorg = oy; h.zorg = oz;
  }
  h_ = h;
  return true;
}

Reader::~Reader() { if (f_) fclose(f_); }

bool Reader::read_slice_f32(int z, std::vector<float> &out, std::string *err) {
  if (z < 0 || z >= h_.nz) { if (err) *err = "slice index out of range"; return false; }
  size_t sb = h_.slice_bytes();
  std::vector<uint8_t> raw(sb);
  if (fseeko(f_, (off_t)(h_.data_offset() + (uint64_t)z * sb), SEEK_SET) != 0 || fread(raw.data(), 1, sb, f_) != sb) {
    if (err) *err = "failed to fill whole buffer";
    return false;
  }
  const bool be = swapped_;
  auto g16 = [&](size_t i) { uint16_t v = be ? (uint16_t)(raw[i] << 8 | raw[i + 1]) : (uint16_t)(raw[i] | raw[i + 1] << 8); return v; };
  auto g32 = [&](size_t i) {
    uint32_t v = be ? ((uint32_t)raw[i] << 24 | (uint32_t)raw[i + 1] << 16 | (uint32_t)raw[i + 2] << 8 | raw[i + 3])
                    : ((uint32_t)raw[i] | (uint32_t)raw[i + 1] << 8 | (uint32_t)raw[i + 2] << 16 | (uint32_t)raw[i + 3] << 24);
    float f; memcpy(&f, &v, 4); return f;
  };
  out.clear();
  const size_t npix = (size_t)h_.nx * h_.ny;
  switch (h_.mode) {
    case BYTE: case RGB: out.assign(raw.begin(), raw.end()); break;
    case SHORT: out.resize(sb / 2); for (size_t i = 0; i < out.size(); ++i) out[i] = (float)(int16_t)g16(2 * i); break;
    case USHORT: out.resize(sb / 2); for (size_t i = 0; i < out.size(); ++i) out[i] = (float)g16(2 * i); break;
    case FLOAT: out.resize(sb / 4); for (size_t i = 0; i < out.size(); ++i) out[i] = g32(4 * i); break;
    case COMPLEX_SHORT:
      out.resize(sb / 4);
      for (size_t i = 0; i < out.size(); ++i) {
        float re = (float)(int16_t)g16(4 * i), im = (float)(int16_t)g16(4 * i + 2);
        out[i] = sqrtf(re * re + im * im);
      }
      break;
    case COMPLEX_FLOAT:
      out.resize(sb / 8);
      for (size_t i = 0; i < out.size(); ++i) {
        float re = g32(8 * i), im = g32(8 * i + 4);
        out[i] = sqrtf(re * re + im * im);
      }
      break;
    case HALF: out.resize(sb / 2); for (size_t i = 0; i < out.size(); ++i) out[i] = f16_to_f32(g16(2 * i)); break;
    case FOURBIT: {
      out.reserve(npix);
      size_t rb = (size_t)(h_.nx + 1) / 2;
      for (int r = 0; r < h_.ny; ++r)
        for (int c = 0; c < h_.nx; ++c) {
          uint8_t byte = raw[r * rb + c / 2];
          out.push_back((float)(c % 2 == 0 ? (byte & 0x0F) : (byte >> 4)));
        }
      break;
    }
    default:
      if (err) *err = "Unsupported MRC mode: " + std::to_string(h_.mode);
      return false;
  }
  return true;
}

// write_slice_raw (write.rs:43-55): the bytes of one section in the file's mode
bool Writer::write_slice_raw(const void *data, size_t bytes, std::string *err) {
  if (bytes != h_.slice_bytes()) {
    if (err) *err = "slice data size " + std::to_string(bytes) + " doesn't match expected " +
                    std::to_string(h_.slice_bytes());
    return false;
  }
  if (fwrite(data, 1, bytes, f_) != bytes) { if (err) *err = "write failed"; return false; }
  return true;
}

bool Writer::create(const std::string &path, const Header &h, std::string *err) {
  f_ = fopen(path.c_str(), "wb");
  if (!f_) { if (err) *err = "cannot create " + path; return false; }
  h_ = h;
  uint8_t b[1024];
  h.to_bytes(b, false);
  if (fwrite(b, 1, 1024, f_) != 1024) { if (err) *err = "write failed"; return false; }
  if (h.next > 0) {
    std::vector<uint8_t> z((size_t)h.next, 0);
    if (fwrite(z.data(), 1, z.size(), f_) != z.size()) { if (err) *err = "write failed"; return false; }
  }
  return true;
}

bool Writer::write_slice_f32(const float *data, size_t n, std::string *err) {
  const size_t npix = (size_t)h_.nx * h_.ny;
  if (n != npix) { if (err) *err = "data length mismatch"; return false; }
  std::vector<uint8_t> buf;
  switch (h_.mode) {
    case BYTE:
      buf.resize(npix);
      for (size_t i = 0; i < npix; ++i) {
        float v = std::min(std::max(data[i], 0.0f), 255.0f);
        buf[i] = (uint8_t)v;
      }
      break;
    case SHORT:
      buf.resize(npix * 2);
      for (size_t i = 0; i < npix; ++i) {
        float v = data[i];  // Rust `as i16` saturates, NaN -> 0
        int16_t s = v != v ? 0 : v >= 32767.0f ? 32767 : v <= -32768.0f ? -32768 : (int16_t)v;
        memcpy(&buf[2 * i], &s, 2);
      }
      break;
    case USHORT:
      buf.resize(npix * 2);
      for (size_t i = 0; i < npix; ++i) {
        float v = std::min(std::max(data[i], 0.0f), 65535.0f);
        uint16_t s = v != v ? 0 : (uint16_t)v;
        memcpy(&buf[2 * i], &s, 2);
      }
      break;
    case FLOAT:
      buf.resize(npix * 4);
      memcpy(buf.data(), data, npix * 4);  // little-endian host
      break;
    case HALF:  // addition: the reference reads mode 12 but does not write it
      buf.resize(npix * 2);
      for (size_t i = 0; i < npix; ++i) {
        const uint16_t hb = f32_to_f16(data[i]);
        memcpy(&buf[2 * i], &hb, 2);
      }
      break;
    default:
      if (err) *err = "Unsupported MRC mode: " + std::to_string(h_.mode);
      return false;
  }
  if (fwrite(buf.data(), 1, buf.size(), f_) != buf.size()) { if (err) *err = "write failed"; return false; }
  return true;
}

bool Writer::finish(float amin, float amax, float amean, std::string *err) {
  h_.amin = amin;
  h_.amax = amax;
  h_.amean = amean;
  uint8_t b[1024];
  h_.to_bytes(b, false);
  if (fseeko(f_, 0, SEEK_SET) != 0 || fwrite(b, 1, 1024, f_) != 1024 || fflush(f_) != 0) {
    if (err) *err = "header rewrite failed";
    return false;
  }
  fclose(f_);
  f_ = nullptr;
  return true;
}

Writer::~Writer() { if (f_) fclose(f_); }

static std::string trim(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && isspace((unsigned char)s[a])) ++a;
  while (b > a && isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

bool parse_f32(const std::string &s, float &out) {
  if (s.empty()) return false;
  for (char c : s)
    if (isspace((unsigned char)c)) return false;
  // Rust accepts decimal/exponent forms, "inf", "infinity", "nan" (any case); no hex
  if (s.find('x') != std::string::npos || s.find('X') != std::string::npos) return false;
  char *end = nullptr;
  errno = 0;
  float v = strtof(s.c_str(), &end);
  if (end != s.c_str() + s.size()) return false;
  out = v;
  return true;
}

bool read_tilt_file(const std::string &path, std::vector<float> &angles, std::string *err) {
  std::ifstream f(path);
  if (!f) { if (err) *err = "No such file or directory (os error 2)"; return false; }
  std::string line;
  angles.clear();
  while (std::getline(f, line)) {
    std::string t = trim(line);
    if (t.empty()) continue;
    float v;
    if (parse_f32(t, v)) angles.push_back(v);
  }
  return true;
}

bool load_per_view_file(const std::string &path, std::vector<float> &vals, std::string *err) {
  std::ifstream f(path);
  if (!f) { if (err) *err = "No such file or directory (os error 2)"; return false; }
  std::string line;
  vals.clear();
  while (std::getline(f, line)) {
    std::string t = trim(line);
    if (t.empty() || t[0] == '#') continue;
    float v;
    if (!parse_f32(t, v)) {
      if (err) *err = "parse error: invalid float literal";
      return false;
    }
    vals.push_back(v);
  }
  return true;
}

bool load_local_rows(const std::string &path, std::vector<float> &rows, std::string *err) {
  std::ifstream f(path);
  if (!f) { if (err) *err = "No such file or directory (os error 2)"; return false; }
  std::string line;
  rows.clear();
  while (std::getline(f, line)) {
    std::string t = trim(line);
    if (t.empty() || t[0] == '#') continue;
    std::istringstream ss(t);
    std::vector<std::string> parts;
    std::string p;
    while (ss >> p) parts.push_back(p);
    if (parts.size() < 5) continue;
    // view: usize parse, 0 on failure
    float view = 0.0f;
    {
      const std::string &s = parts[0];
      bool ok = !s.empty();
      size_t i = (s[0] == '+') ? 1 : 0;
      if (i >= s.size()) ok = false;
      for (size_t k = i; k < s.size() && ok; ++k) ok = isdigit((unsigned char)s[k]) != 0;
      if (ok) view = (float)strtoull(s.c_str() + i, nullptr, 10);
    }
    rows.push_back(view);
    for (int k = 1; k < 5; ++k) {
      float v = 0.0f;
      if (!parse_f32(parts[k], v)) v = 0.0f;
      rows.push_back(v);
    }
  }
  return true;
}

}  // namespace mrc
