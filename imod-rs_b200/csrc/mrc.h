// mrc.h -- MRC 2014 file format, byte-compatible with crates/imod-mrc.
//
// Header layout: crates/imod-mrc/src/header.rs:10-110 (1024 bytes, written
// little-endian).  Reader: crates/imod-mrc/src/read.rs:28-231 (byte-swap
// detection by machine stamp or unreasonable dimensions, old-style origin
// fix-up, extended header skip, every mode converted to f32).  Writer:
// crates/imod-mrc/src/write.rs:20-153 (header, zeroed extended header,
// slices, header rewritten with statistics on finish).
#pragma once
#include <stdint.h>

#include <cstdio>
#include <string>
#include <vector>

namespace mrc {

enum Mode { BYTE = 0, SHORT = 1, FLOAT = 2, COMPLEX_SHORT = 3, COMPLEX_FLOAT = 4, USHORT = 6,
            HALF = 12, RGB = 16, FOURBIT = 101 };

struct Header {
  int32_t nx = 0, ny = 0, nz = 0, mode = 0;
  int32_t nxstart = 0, nystart = 0, nzstart = 0;
  int32_t mx = 0, my = 0, mz = 0;
  float xlen = 0, ylen = 0, zlen = 0;
  float alpha = 90, beta = 90, gamma = 90;
  int32_t mapc = 1, mapr = 2, maps = 3;
  float amin = 0, amax = 0, amean = 0;
  int32_t ispg = 0, next = 0;
  int16_t creatid = 0;
  uint8_t blank[6] = {0};
  uint8_t ext_type[4] = {0};
  int32_t nversion = 20140;
  uint8_t blank2[16] = {0};
  int16_t nint = 0, nreal = 0, sub = 0, zfac = 0;
  float min2 = 0, max2 = 0, min3 = 0, max3 = 0;
  int32_t imod_stamp = 0, imod_flags = 0;
  int16_t idtype = 0, lens = 0, nd1 = 0, nd2 = 0, vd1 = 0, vd2 = 0;
  float tilt_angles[6] = {0};
  float xorg = 0, yorg = 0, zorg = 0;
  uint8_t cmap[4] = {'M', 'A', 'P', ' '};
  uint8_t stamp[4] = {0x44, 0x44, 0, 0};
  float rms = -1.0f;
  int32_t nlabl = 0;
  char labels[10][80] = {{0}};

  static constexpr int32_t IMOD_STAMP = (int32_t)0x25004488u;
  // MrcHeader::new (header.rs:181-241)
  static Header make(int32_t nx, int32_t ny, int32_t nz, int32_t mode);
  // add_label (header.rs:244-258): copy up to 80 bytes, pad with spaces
  bool add_label(const std::string &text);
  std::string label(int idx) const;
  bool is_swapped() const { return stamp[0] == 0x11 && stamp[1] == 0x11; }
  bool is_old_style() const;
  size_t slice_bytes() const;
  uint64_t data_offset() const { return 1024 + (uint64_t)(next > 0 ? next : 0); }
  int bytes_per_pixel() const;
  // serialise / parse the 1024 on-disk bytes
  void to_bytes(uint8_t out[1024], bool big_endian = false) const;
  static Header from_bytes(const uint8_t in[1024], bool big_endian);
};

class Reader {
 public:
  bool open(const std::string &path, std::string *err);
  const Header &header() const { return h_; }
  bool swapped() const { return swapped_; }
  // read_slice_f32 (read.rs:127-231); RGB yields 3 values per pixel as in the reference
  bool read_slice_f32(int z, std::vector<float> &out, std::string *err);
  ~Reader();

 private:
  FILE *f_ = nullptr;
  Header h_;
  bool swapped_ = false;
};

class Writer {
 public:
  bool create(const std::string &path, const Header &h, std::string *err);
  // write_slice_f32 (write.rs:58-104), plus mode 12 (IEEE half, round to nearest even)
  bool write_slice_f32(const float *data, size_t n, std::string *err);
  bool write_slice_raw(const void *data, size_t bytes, std::string *err);
  bool finish(float amin, float amax, float amean, std::string *err);
  ~Writer();

 private:
  FILE *f_ = nullptr;
  Header h_;
};

float f16_to_f32(uint16_t bits);
uint16_t f32_to_f16(float f);

// read_tilt_file (crates/imod-transforms/src/tilt.rs:6-23)
bool read_tilt_file(const std::string &path, std::vector<float> &angles, std::string *err);
// load_per_view_file (apps/tilt/src/main.rs:310-326)
bool load_per_view_file(const std::string &path, std::vector<float> &vals, std::string *err);
// load_local_alignment's parsing (apps/tilt/src/main.rs:232-253): rows of 5 floats
bool load_local_rows(const std::string &path, std::vector<float> &rows, std::string *err);
// f32 parse with Rust's str::parse::<f32> acceptance (whole string, no spaces)
bool parse_f32(const std::string &s, float &out);

}  // namespace mrc
