// studio.cpp -- imod-studio's reconstruction step on the B200 path.
//
// step_reconstruction (apps/imod-studio/src/main.rs:725-776) reads <base>.ali
// and <base>.tlt, back-projects every row without R-weighting or cosine
// stretch (zero fill, thickness = width, x = ((ox-cx)*cos + (oz-cz)*sin) + cx,
// sum / nz) and writes <base>_full.rec with the label
// "imod-studio: reconstruction" and header statistics (0, 0, 0).  That is the
// tilt path with --no-weight --no-cosine-stretch --fill-mode zero -z <width>,
// so this file only maps the step onto a session and the MRC boundary.
#include <string.h>
#include <sys/stat.h>

#include <string>
#include <vector>

#include "mrc.h"
#include "tiltgpu.h"

namespace tg {
void set_error(const std::string &m);
}

namespace {
bool exists(const char *p) {
  struct stat st;
  return stat(p, &st) == 0;
}
}  // namespace

extern "C" int tg_studio_reconstruct(const char *ali_path, const char *tlt_path, const char *rec_path,
                                     int32_t device) {
  if (!ali_path || !tlt_path || !rec_path) return TG_ERR_INVALID_ARG;
  // the step's own checks, in its order (main.rs:730-731)
  if (!exists(ali_path)) { tg::set_error(std::string(ali_path) + " not found"); return TG_ERR_INVALID_ARG; }
  if (!exists(tlt_path)) { tg::set_error(std::string(tlt_path) + " not found"); return TG_ERR_INVALID_ARG; }
  std::string err;
  std::vector<float> angles;
  if (!mrc::read_tilt_file(tlt_path, angles, &err)) { tg::set_error(err); return TG_ERR_INVALID_ARG; }
  mrc::Reader reader;
  if (!reader.open(ali_path, &err)) { tg::set_error(err); return TG_ERR_INVALID_ARG; }
  const mrc::Header h = reader.header();
  const int in_nx = h.nx, in_ny = h.ny, nz = h.nz, out_nz = in_nx;
  std::vector<float> proj((size_t)in_nx * in_ny * nz), sl;
  for (int z = 0; z < nz; ++z) {
    if (!reader.read_slice_f32(z, sl, &err) || sl.size() != (size_t)in_nx * in_ny) {
      tg::set_error(err.empty() ? "unsupported slice layout" : err);
      return TG_ERR_INVALID_ARG;
    }
    memcpy(proj.data() + (size_t)z * in_nx * in_ny, sl.data(), sl.size() * sizeof(float));
  }
  tg_geometry g{};
  g.nx = in_nx;
  g.ny = in_ny;
  g.nz = nz;
  g.out_nx = in_nx;
  g.out_nz = out_nz;
  g.n_angles = (int32_t)angles.size();
  g.angles = angles.data();
  tg_options o;
  tg_options_default(&o);
  o.no_weight = 1;
  o.no_cosine_stretch = 1;
  o.fill_mode = TG_FILL_ZERO;
  o.device = device;
  tg_session *s = nullptr;
  int rc = tg_session_create(&g, &o, &s);
  if (rc != TG_OK) return rc;
  std::vector<float> vol((size_t)in_ny * out_nz * in_nx);
  if ((rc = tg_upload_projections(s, proj.data(), proj.size())) != TG_OK || (rc = tg_reconstruct(s)) != TG_OK ||
      (rc = tg_download_slices(s, 0, in_ny, vol.data(), nullptr)) != TG_OK) {
    tg_session_destroy(s);
    return rc;
  }
  tg_session_destroy(s);
  // MrcHeader::new(in_nx, out_nz, in_ny, Float) + the step's label; finish(0, 0, 0)
  mrc::Header oh = mrc::Header::make(in_nx, out_nz, in_ny, mrc::FLOAT);
  oh.add_label("imod-studio: reconstruction");
  mrc::Writer w;
  if (!w.create(rec_path, oh, &err)) { tg::set_error(err); return TG_ERR_INVALID_ARG; }
  const size_t slice = (size_t)in_nx * out_nz;
  for (int iy = 0; iy < in_ny; ++iy)
    if (!w.write_slice_f32(vol.data() + (size_t)iy * slice, slice, &err)) { tg::set_error(err); return TG_ERR_INVALID_ARG; }
  if (!w.finish(0.0f, 0.0f, 0.0f, &err)) { tg::set_error(err); return TG_ERR_INVALID_ARG; }
  return TG_OK;
}
