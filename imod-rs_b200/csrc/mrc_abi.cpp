// mrc_abi.cpp -- C ABI over the MRC and tilt-file code (host only).
#include <string.h>

#include <cstdio>
#include <string>
#include <vector>

#include "mrc.h"
#include "tiltgpu.h"

namespace tg {
void set_error(const std::string &m);
}

extern "C" {

int tg_mrc_header_new(int32_t nx, int32_t ny, int32_t nz, int32_t mode, const char *label, uint8_t out[1024]) {
  if (!out) return TG_ERR_INVALID_ARG;
  mrc::Header h = mrc::Header::make(nx, ny, nz, mode);
  if (label) h.add_label(label);
  h.to_bytes(out, false);
  return TG_OK;
}

int tg_mrc_read(const char *path, tg_mrc_info *info, int32_t z0, int32_t z1, float *out) {
  if (!path) return TG_ERR_INVALID_ARG;
  mrc::Reader r;
  std::string err;
  if (!r.open(path, &err)) { tg::set_error(err); return TG_ERR_INVALID_ARG; }
  const mrc::Header &h = r.header();
  if (info) {
    info->nx = h.nx; info->ny = h.ny; info->nz = h.nz; info->mode = h.mode; info->next = h.next;
    info->swapped = r.swapped();
    info->xlen = h.xlen; info->ylen = h.ylen; info->zlen = h.zlen;
    info->amin = h.amin; info->amax = h.amax; info->amean = h.amean;
    info->nlabl = h.nlabl;
    info->imod = h.imod_stamp == mrc::Header::IMOD_STAMP;
    h.to_bytes(info->header, false);
  }
  if (!out) return TG_OK;
  if (z0 < 0 || z1 > h.nz || z0 > z1) return TG_ERR_INVALID_ARG;
  std::vector<float> sl;
  size_t off = 0;
  for (int z = z0; z < z1; ++z) {
    if (!r.read_slice_f32(z, sl, &err)) { tg::set_error(err); return TG_ERR_INVALID_ARG; }
    memcpy(out + off, sl.data(), sl.size() * 4);
    off += sl.size();
  }
  return TG_OK;
}

int tg_mrc_write_f32(const char *path, const uint8_t header[1024], const float *data, int32_t nsec,
                     float amin, float amax, float amean) {
  if (!path || !header || (nsec > 0 && !data)) return TG_ERR_INVALID_ARG;
  mrc::Header h = mrc::Header::from_bytes(header, false);
  mrc::Writer w;
  std::string err;
  if (!w.create(path, h, &err)) { tg::set_error(err); return TG_ERR_INVALID_ARG; }
  size_t n = (size_t)h.nx * h.ny;
  for (int z = 0; z < nsec; ++z)
    if (!w.write_slice_f32(data + (size_t)z * n, n, &err)) { tg::set_error(err); return TG_ERR_INVALID_ARG; }
  if (!w.finish(amin, amax, amean, &err)) { tg::set_error(err); return TG_ERR_INVALID_ARG; }
  return TG_OK;
}

int tg_tilt_output_header(const uint8_t in_header[1024], int32_t out_nx, int32_t out_nz, uint8_t out[1024]) {
  if (!in_header || !out) return TG_ERR_INVALID_ARG;
  mrc::Header h = mrc::Header::from_bytes(in_header, false);
  if (h.nx <= 0 || out_nx <= 0 || out_nz <= 0) return TG_ERR_INVALID_ARG;
  const int out_ny = h.ny;
  mrc::Header oh = mrc::Header::make(out_nx, out_nz, out_ny, mrc::FLOAT);
  oh.xlen = h.xlen * (float)out_nx / (float)h.nx;
  oh.ylen = h.xlen * (float)out_nz / (float)h.nx;
  oh.zlen = h.ylen;
  oh.mx = out_nx;
  oh.my = out_nz;
  oh.mz = out_ny;
  oh.add_label("tilt: " + std::to_string(h.nz) + " projections, thickness " + std::to_string(out_nz));
  oh.to_bytes(out, false);
  return TG_OK;
}

int tg_read_tilt_file(const char *path, float *out, int32_t cap, int32_t *n) {
  if (!path || !n) return TG_ERR_INVALID_ARG;
  std::vector<float> a;
  std::string err;
  if (!mrc::read_tilt_file(path, a, &err)) { tg::set_error(err); return TG_ERR_INVALID_ARG; }
  *n = (int32_t)a.size();
  for (int i = 0; i < (int)a.size() && i < cap && out; ++i) out[i] = a[i];
  return TG_OK;
}

int tg_write_tilt_file(const char *path, const float *angles, int32_t n) {
  if (!path || (n > 0 && !angles)) return TG_ERR_INVALID_ARG;
  FILE *f = fopen(path, "w");
  if (!f) { tg::set_error("cannot create file"); return TG_ERR_INVALID_ARG; }
  for (int i = 0; i < n; ++i) fprintf(f, "%10.2f\n", (double)angles[i]);  // "{:10.2}"
  fclose(f);
  return TG_OK;
}

}  // extern "C"
