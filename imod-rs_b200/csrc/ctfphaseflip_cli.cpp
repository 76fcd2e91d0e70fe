// ctfphaseflip_cli.cpp -- drop-in `ctfphaseflip`: the reference's command line
// (clap Args of apps/ctfphaseflip/src/main.rs:19-88), its defocus-file parsing
// and interpolation (94-209), MRC in/out through the same byte-compatible
// reader and writer as `tilt`, and the whole correction on the GPU through
// tg_ctf_phaseflip.  Additions: --device N selects the GPU; --gpu is accepted
// (every strip is corrected on the GPU either way).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "mrc.h"
#include "tiltgpu.h"

namespace {

struct Args {
  std::string input, output, tilt_file, defocus_file;
  float defocus = -3000.0f, voltage = 300.0f, cs = 2.7f;
  bool has_pixel = false;
  float pixel_size = 0.0f;
  long strip_width = 256;
  float tilt_axis_angle = 0.0f;
  long max_strip_width = 0;  // 0: not given
  float amplitude_contrast = 0.07f, cuton_freq = 0.0f, plate_phase = 0.0f;
  bool gpu = false;
  int device = 0;
};

void usage(FILE *f) {
  fprintf(f,
          "CTF phase-flip correction of a tilt series (B200)\n\n"
          "Usage: ctfphaseflip [OPTIONS] --input <INPUT> --output <OUTPUT> --tilt-file <TILT_FILE>\n\n"
          "Options:\n"
          "  -i, --input <INPUT>                    Input tilt series MRC file\n"
          "  -o, --output <OUTPUT>                  Output corrected MRC file\n"
          "  -t, --tilt-file <TILT_FILE>            Tilt angle file (.tlt)\n"
          "  -d, --defocus <DEFOCUS>                Defocus in nm (negative = underfocus) [default: -3000]\n"
          "      --defocus-file <DEFOCUS_FILE>      Lines \"view defocus1 [defocus2 astig_angle]\" (nm, deg)\n"
          "  -v, --voltage <VOLTAGE>                Voltage in kV [default: 300]\n"
          "  -c, --cs <CS>                          Spherical aberration in mm [default: 2.7]\n"
          "  -p, --pixel-size <PIXEL_SIZE>          Pixel size in Angstroms (overrides header)\n"
          "  -w, --strip-width <STRIP_WIDTH>        Width of strips in pixels [default: 256]\n"
          "      --tilt-axis-angle <DEG>            Tilt axis rotation from Y, degrees [default: 0]\n"
          "      --max-strip-width <N>              Maximum strip width (default: from defocus and pixel)\n"
          "      --amplitude-contrast <W>           Amplitude contrast fraction [default: 0.07]\n"
          "      --cuton-freq <F>                   No correction below this frequency (1/A) [default: 0]\n"
          "      --gpu                              Accepted; the correction always runs on the GPU\n"
          "      --plate-phase <DEG>                Phase plate phase shift in degrees [default: 0]\n"
          "      --device <N>                       CUDA device ordinal (addition)\n"
          "  -h, --help                             Print help\n");
}

[[noreturn]] void clap_error(const std::string &msg) {
  fprintf(stderr, "error: %s\n\nFor more information, try '--help'.\n", msg.c_str());
  exit(2);
}

long parse_uint(const std::string &v, const std::string &flag) {
  char *end = nullptr;
  errno = 0;
  const char *s = v.c_str() + (v.size() > 1 && v[0] == '+' ? 1 : 0);
  long x = strtol(s, &end, 10);
  if (v.empty() || !isdigit((unsigned char)*s) || *end != '\0' || errno || x < 0)
    clap_error("invalid value '" + v + "' for '" + flag + "': invalid digit found in string");
  return x;
}
float parse_float(const std::string &v, const std::string &flag) {
  float x;
  if (!mrc::parse_f32(v, x)) clap_error("invalid value '" + v + "' for '" + flag + "': invalid float literal");
  return x;
}

Args parse(int argc, char **argv) {
  Args a;
  bool has_in = false, has_out = false, has_tlt = false;
  std::map<std::string, std::string> alias = {
      {"-i", "input"}, {"-o", "output"}, {"-t", "tilt-file"}, {"-d", "defocus"},
      {"-v", "voltage"}, {"-c", "cs"}, {"-p", "pixel-size"}, {"-w", "strip-width"}};
  for (int i = 1; i < argc; ++i) {
    std::string arg = argv[i], val, name;
    bool has_eq = false;
    if (arg == "-h" || arg == "--help") { usage(stdout); exit(0); }
    if (arg.rfind("--", 0) == 0) {
      const size_t eq = arg.find('=');
      if (eq != std::string::npos) { val = arg.substr(eq + 1); arg = arg.substr(0, eq); has_eq = true; }
      name = arg.substr(2);
    } else if (arg.size() >= 2 && arg[0] == '-' && alias.count(arg.substr(0, 2))) {
      name = alias[arg.substr(0, 2)];
      if (arg.size() > 2) { val = arg.substr(2); has_eq = true; }
    } else {
      clap_error("unexpected argument '" + arg + "' found");
    }
    if (name == "gpu") {
      if (has_eq) clap_error("unexpected value '" + val + "' for '--gpu' found; no more were expected");
      a.gpu = true;
      continue;
    }
    static const char *known[] = {"input", "output", "tilt-file", "defocus", "defocus-file", "voltage", "cs",
                                  "pixel-size", "strip-width", "tilt-axis-angle", "max-strip-width",
                                  "amplitude-contrast", "cuton-freq", "plate-phase", "device"};
    if (std::find_if(std::begin(known), std::end(known), [&](const char *k) { return name == k; }) == std::end(known))
      clap_error("unexpected argument '--" + name + "' found");
    if (!has_eq) {
      if (i + 1 >= argc) clap_error("a value is required for '--" + name + "' but none was supplied");
      val = argv[++i];
    }
    if (name == "input") { a.input = val; has_in = true; }
    else if (name == "output") { a.output = val; has_out = true; }
    else if (name == "tilt-file") { a.tilt_file = val; has_tlt = true; }
    else if (name == "defocus") a.defocus = parse_float(val, "--defocus");
    else if (name == "defocus-file") a.defocus_file = val;
    else if (name == "voltage") a.voltage = parse_float(val, "--voltage");
    else if (name == "cs") a.cs = parse_float(val, "--cs");
    else if (name == "pixel-size") { a.pixel_size = parse_float(val, "--pixel-size"); a.has_pixel = true; }
    else if (name == "strip-width") a.strip_width = parse_uint(val, "--strip-width");
    else if (name == "tilt-axis-angle") a.tilt_axis_angle = parse_float(val, "--tilt-axis-angle");
    else if (name == "max-strip-width") a.max_strip_width = parse_uint(val, "--max-strip-width");
    else if (name == "amplitude-contrast") a.amplitude_contrast = parse_float(val, "--amplitude-contrast");
    else if (name == "cuton-freq") a.cuton_freq = parse_float(val, "--cuton-freq");
    else if (name == "plate-phase") a.plate_phase = parse_float(val, "--plate-phase");
    else if (name == "device") a.device = (int)parse_uint(val, "--device");
  }
  std::string missing;
  if (!has_in) missing += "\n  --input <INPUT>";
  if (!has_out) missing += "\n  --output <OUTPUT>";
  if (!has_tlt) missing += "\n  --tilt-file <TILT_FILE>";
  if (!missing.empty()) clap_error("the following required arguments were not provided:" + missing);
  return a;
}

struct ViewDefocus { float d1, d2, astig; };

std::string trim(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && isspace((unsigned char)s[a])) ++a;
  while (b > a && isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

// read_defocus_file (main.rs:101-156)
bool read_defocus_file(const std::string &path, std::vector<ViewDefocus> &e, std::vector<size_t> &views,
                       std::string &err) {
  std::ifstream f(path);
  if (!f) { err = "Cannot read defocus file " + path + ": " + strerror(errno); return false; }
  std::string raw;
  int line_num = 0;
  while (std::getline(f, raw)) {
    ++line_num;
    if (!raw.empty() && raw.back() == '\r') raw.pop_back();
    const std::string line = trim(raw);
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ss(line);
    std::vector<std::string> fl;
    for (std::string t; ss >> t;) fl.push_back(t);
    const std::string ln = std::to_string(line_num);
    if (fl.size() < 2) { err = "Defocus file line " + ln + ": expected at least 'view defocus1', got '" + line + "'"; return false; }
    const std::string &v0 = fl[0];
    const size_t digits0 = v0.size() > 1 && v0[0] == '+' ? 1 : 0;
    bool ok = v0.size() > digits0;
    for (size_t k = digits0; k < v0.size(); ++k) ok &= isdigit((unsigned char)v0[k]) != 0;
    if (!ok) { err = "Defocus file line " + ln + ": invalid view number '" + v0 + "'"; return false; }
    const size_t view = (size_t)strtoull(v0.c_str() + digits0, nullptr, 10);
    ViewDefocus d{};
    if (!mrc::parse_f32(fl[1], d.d1)) { err = "Defocus file line " + ln + ": invalid defocus1 '" + fl[1] + "'"; return false; }
    if (fl.size() >= 4) {
      if (!mrc::parse_f32(fl[2], d.d2)) { err = "Defocus file line " + ln + ": invalid defocus2 '" + fl[2] + "'"; return false; }
      if (!mrc::parse_f32(fl[3], d.astig)) { err = "Defocus file line " + ln + ": invalid astig_angle '" + fl[3] + "'"; return false; }
    } else if (fl.size() == 3) {
      if (!mrc::parse_f32(fl[2], d.d2)) { err = "Defocus file line " + ln + ": invalid defocus2 '" + fl[2] + "'"; return false; }
      d.astig = 0.0f;
    } else {
      d.d2 = d.d1;
      d.astig = 0.0f;
    }
    views.push_back(view);
    e.push_back(d);
  }
  return true;
}

// interpolate_defocus (main.rs:162-209): f32 linear interpolation between the
// nearest listed views, the nearest one's values past either end
std::vector<ViewDefocus> interpolate_defocus(const std::vector<ViewDefocus> &e, const std::vector<size_t> &views,
                                             size_t n) {
  if (e.empty() || n == 0) return {};
  std::vector<ViewDefocus> r(n, ViewDefocus{0.0f, 0.0f, 0.0f});
  std::vector<bool> has(n, false);
  for (size_t i = 0; i < e.size(); ++i)
    if (views[i] < n) { r[views[i]] = e[i]; has[views[i]] = true; }
  for (size_t v = 0; v < n; ++v) {
    if (has[v]) continue;
    long b = -1, a = -1;
    for (long i = (long)v - 1; i >= 0; --i) if (has[i]) { b = i; break; }
    for (size_t i = v + 1; i < n; ++i) if (has[i]) { a = (long)i; break; }
    if (b >= 0 && a >= 0) {
      const float t = (float)(v - b) / (float)(a - b);
      r[v].d1 = r[b].d1 + t * (r[a].d1 - r[b].d1);
      r[v].d2 = r[b].d2 + t * (r[a].d2 - r[b].d2);
      r[v].astig = r[b].astig + t * (r[a].astig - r[b].astig);
    } else if (b >= 0) {
      r[v] = r[b];
    } else if (a >= 0) {
      r[v] = r[a];
    }
  }
  return r;
}

}  // namespace

int main(int argc, char **argv) {
  Args args = parse(argc, argv);
  std::string err;
  std::vector<float> angles;
  if (!mrc::read_tilt_file(args.tilt_file, angles, &err)) {  // main.rs:224-227
    fprintf(stderr, "Error reading tilt file: %s\n", err.c_str());
    return 1;
  }
  std::vector<ViewDefocus> entries;
  std::vector<size_t> views;
  const bool has_def_file = !args.defocus_file.empty();
  if (has_def_file && !read_defocus_file(args.defocus_file, entries, views, err)) {  // main.rs:230-235
    fprintf(stderr, "Error: %s\n", err.c_str());
    return 1;
  }
  mrc::Reader reader;
  if (!reader.open(args.input, &err)) {  // main.rs:237-240
    fprintf(stderr, "Error: %s\n", err.c_str());
    return 1;
  }
  const mrc::Header h = reader.header();
  const int nx = h.nx, ny = h.ny, nz = h.nz;
  const float pixel_a = args.has_pixel ? args.pixel_size : (h.mx > 0 ? h.xlen / (float)h.mx : 1.0f);
  std::vector<ViewDefocus> vd;
  if (has_def_file) {
    if (entries.size() < (size_t)nz)
      fprintf(stderr, "ctfphaseflip: defocus file has %zu entries for %d views, interpolating missing values\n",
              entries.size(), nz);
    vd = interpolate_defocus(entries, views, (size_t)nz);
  }
  if (angles.size() < (size_t)nz)
    fprintf(stderr, "Warning: tilt file has %zu angles but stack has %d sections\n", angles.size(), nz);
  tg_ctf_options o;
  tg_ctf_options_default(&o);
  o.defocus = args.defocus;
  o.voltage = args.voltage;
  o.cs = args.cs;
  o.pixel_size = pixel_a;
  o.strip_width = (int32_t)args.strip_width;
  o.tilt_axis_angle = args.tilt_axis_angle;
  o.max_strip_width = (int32_t)args.max_strip_width;
  o.amplitude_contrast = args.amplitude_contrast;
  o.cuton_freq = args.cuton_freq;
  o.plate_phase = args.plate_phase;
  o.device = args.device;
  std::vector<float> vdf;
  for (const auto &d : vd) { vdf.push_back(d.d1); vdf.push_back(d.d2); vdf.push_back(d.astig); }
  static float empty_marker[3];  // a defocus file without entries: given, but no per-view values
  const float *vdp = has_def_file ? (vdf.empty() ? empty_marker : vdf.data()) : nullptr;
  int32_t strip_w = 0;
  tg_ctf_strip_width(&o, nx, vdp, (int32_t)vd.size(), &strip_w);
  fprintf(stderr, "ctfphaseflip: voltage=%.0fkV, Cs=%.1fmm, pixel=%.2fA, strips=%dpx, tilt_axis=%.1fdeg (B200)\n",
          (double)args.voltage, (double)args.cs, (double)pixel_a, strip_w, (double)args.tilt_axis_angle);
  if (fabsf(args.plate_phase) > 1e-6f)
    fprintf(stderr, "ctfphaseflip: phase plate correction=%.1fdeg\n", (double)args.plate_phase);
  if (has_def_file) fprintf(stderr, "ctfphaseflip: using per-view defocus file with astigmatism support\n");
  else fprintf(stderr, "ctfphaseflip: defocus=%.0fnm\n", (double)args.defocus);
  // output header (main.rs:348-355)
  mrc::Header oh = mrc::Header::make(h.nx, h.ny, h.nz, mrc::FLOAT);
  oh.xlen = h.xlen;
  oh.ylen = h.ylen;
  oh.zlen = h.zlen;
  oh.mx = h.mx;
  oh.my = h.my;
  oh.mz = h.mz;
  oh.add_label("ctfphaseflip: CTF phase correction (2D strips)");
  const size_t sec = (size_t)nx * ny;
  std::vector<float> in(sec * nz), out(sec * nz), sl;
  for (int z = 0; z < nz; ++z) {
    if (!reader.read_slice_f32(z, sl, &err) || sl.size() != sec) {
      fprintf(stderr, "Error: %s\n", err.empty() ? "unsupported slice layout" : err.c_str());
      return 1;
    }
    std::copy(sl.begin(), sl.end(), in.begin() + (size_t)z * sec);
  }
  tg_stats st{};
  const int rc = tg_ctf_phaseflip(&o, in.data(), nx, ny, nz, angles.data(), (int32_t)angles.size(), vdp,
                                  (int32_t)vd.size(), out.data(), &st);
  if (rc != TG_OK) {
    fprintf(stderr, "Error: %s (%s)\n", tg_status_string(rc), tg_last_error());
    return 1;
  }
  mrc::Writer w;
  if (!w.create(args.output, oh, &err)) { fprintf(stderr, "Error: %s\n", err.c_str()); return 1; }
  for (int z = 0; z < nz; ++z)
    if (!w.write_slice_f32(out.data() + (size_t)z * sec, sec, &err)) { fprintf(stderr, "Error: %s\n", err.c_str()); return 1; }
  if (!w.finish(st.amin, st.amax, st.amean, &err)) { fprintf(stderr, "Error: %s\n", err.c_str()); return 1; }
  fprintf(stderr, "ctfphaseflip: corrected %d sections (2D strips)\n", nz);
  return 0;
}
