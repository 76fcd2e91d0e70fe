// tilt_cli.cpp -- drop-in `tilt`: the reference's command line (clap Args of
// apps/tilt/src/main.rs:18-120) plus IMOD PIP-style aliases, MRC in/out
// byte-compatible with crates/imod-mrc, and the whole reconstruction on the
// GPU through libtiltgpu's C ABI.
//
// Additions beyond the reference (documented in --help): the PIP aliases
// -InputProjections -OutputFile -TILTFILE -THICKNESS -WIDTH -RADIAL
// -SIRTIterations -LOG -SCALE -FakeSIRTiterations -XAXISTILT-file aliases are
// mapped onto the same fields; --storage fp32|fp16|bf16 and --device N select
// the staging precision and GPU.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cctype>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

#include "mrc.h"
#include "tiltgpu.h"

namespace {

struct Args {
  std::string input, output, tilt_file;
  int thickness = 0;
  bool has_width = false;
  int width = 0;
  long threads = -1;
  bool gpu = false;
  std::string radial = "0.35,0.05";
  bool no_weight = false;
  long sirt = 0;
  float sirt_relax = 1.0f;
  bool no_cosine_stretch = false;
  std::string local_file, xtilt_file, zfactor_file;
  bool log = false;
  float densweight = 1.0f, outscale = 1.0f, outadd = 0.0f;
  long exact_filter_size = 0;
  std::string fill_mode = "mean", cosine_interp = "linear";
  float max_cosine_tilt = 80.0f;
  bool hamming = false;
  bool exact_xtilt = false;
  long fake_sirt = 0;
  std::string storage = "fp32";
  int device = 0;
  int mode = 2;  // output MRC mode: 2 (float, the reference's) or 12 (half)
  long io_chunk_kb = 128 * 1024;  // pinned staging chunk of the read and write pipelines
  std::string checkpoint, resume;  // SIRT state files (MRC, iteration count in the first label)
  long checkpoint_every = 10;
};

void usage(FILE *f) {
  fprintf(f,
          "Weighted back-projection reconstruction (B200)\n\n"
          "Usage: tilt [OPTIONS] --input <INPUT> --output <OUTPUT> --tilt-file <TILT_FILE>\n\n"
          "Options:\n"
          "  -i, --input <INPUT>              Input aligned tilt series (MRC)\n"
          "  -o, --output <OUTPUT>            Output reconstruction (MRC)\n"
          "  -t, --tilt-file <TILT_FILE>      Tilt angle file (.tlt)\n"
          "  -z, --thickness <THICKNESS>      Thickness of output volume in Z (pixels) [default: 0]\n"
          "  -w, --width <WIDTH>              Width of output (default: same as input)\n"
          "  -j, --threads <THREADS>          Accepted for compatibility (all work is on the GPU)\n"
          "      --gpu                        Semantics of the reference's wgpu back-projector\n"
          "      --radial <RADIAL>            R-weighting cutoff,falloff [default: 0.35,0.05]\n"
          "      --no-weight                  Disable R-weighting filter\n"
          "      --sirt <SIRT>                Number of SIRT iterations (0 = plain WBP) [default: 0]\n"
          "      --sirt-relax <SIRT_RELAX>    SIRT relaxation factor [default: 1]\n"
          "      --no-cosine-stretch          Disable cosine stretching of projections\n"
          "      --local-file <LOCAL_FILE>    Local alignment file (view x y dx dy per line)\n"
          "      --xtilt-file <XTILT_FILE>    X-axis tilt file (one angle in degrees per view)\n"
          "      --zfactor-file <ZFACTOR_FILE> Per-view Z scaling factor file\n"
          "      --log                        Apply log10 to projection values first\n"
          "      --densweight <DENSWEIGHT>    Density weight factor [default: 1]\n"
          "      --outscale <OUTSCALE>        Output scale factor [default: 1]\n"
          "      --outadd <OUTADD>            Output additive offset [default: 0]\n"
          "      --exact-filter-size <N>      Radial filter table size\n"
          "      --fill-mode <FILL_MODE>      mean, zero or edge [default: mean]\n"
          "      --cosine-interp <MODE>       linear or cubic [default: linear]\n"
          "      --max-cosine-tilt <DEG>      Max tilt for cosine stretching [default: 80]\n"
          "      --hamming                    Hamming window instead of Gaussian rolloff\n"
          "      --fake-sirt <N>              Low-pass smoothing passes [default: 0]\n"
          "      --storage <fp32|fp16|bf16>   Staging precision of filtered projections (addition)\n"
          "      --device <N>                 CUDA device ordinal (addition)\n"
          "      --exact-xtilt                Per-view x-tilt row blend, bit-identical (addition)\n"
          "      --mode <2|12>                Output MRC mode: 2 float, 12 half (addition) [default: 2]\n"
          "      --io-chunk-kb <N>            Staging chunk of the overlapped read/write (addition)\n"
          "                                   [default: 131072]\n"
          "      --checkpoint <FILE>          Write the SIRT state (raw volume, iteration count) to\n"
          "                                   FILE every --checkpoint-every iterations (addition)\n"
          "      --checkpoint-every <K>       [default: 10]\n"
          "      --resume <FILE>              Continue SIRT from a --checkpoint file (addition)\n"
          "  -h, --help                       Print help\n\n"
          "PIP-style aliases (additions): -InputProjections -OutputFile -TILTFILE -THICKNESS\n"
          "  -WIDTH -RADIAL -SIRTIterations -LOG -SCALE <add,mult> -FakeSIRTiterations\n"
          "  -XTILTFILE -ZFACTORFILE -LOCALFILE -HAMMING\n");
}

[[noreturn]] void clap_error(const std::string &msg) {
  fprintf(stderr, "error: %s\n\nFor more information, try '--help'.\n", msg.c_str());
  exit(2);
}

long parse_int(const std::string &v, const std::string &flag, bool allow_neg) {
  char *end = nullptr;
  errno = 0;
  long x = strtol(v.c_str(), &end, 10);
  if (v.empty() || end != v.c_str() + v.size() || errno || (!allow_neg && x < 0))
    clap_error("invalid value '" + v + "' for '" + flag + "': invalid digit found in string");
  return x;
}
float parse_float(const std::string &v, const std::string &flag) {
  float x;
  if (!mrc::parse_f32(v, x)) clap_error("invalid value '" + v + "' for '" + flag + "': invalid float literal");
  return x;
}

std::string lower(std::string s) {
  for (auto &c : s) c = (char)tolower((unsigned char)c);
  return s;
}

Args parse(int argc, char **argv) {
  Args a;
  bool has_in = false, has_out = false, has_tlt = false;
  // long flag -> canonical name; PIP aliases (case-insensitive) map here too
  std::map<std::string, std::string> alias = {
      {"-i", "input"}, {"--input", "input"}, {"-o", "output"}, {"--output", "output"},
      {"-t", "tilt-file"}, {"--tilt-file", "tilt-file"}, {"-z", "thickness"}, {"--thickness", "thickness"},
      {"-w", "width"}, {"--width", "width"}, {"-j", "threads"}, {"--threads", "threads"}};
  std::map<std::string, std::string> pip = {
      {"inputprojections", "input"}, {"inputfile", "input"}, {"outputfile", "output"},
      {"tiltfile", "tilt-file"}, {"thickness", "thickness"}, {"width", "width"}, {"radial", "radial"},
      {"sirtiterations", "sirt"}, {"log", "LOG"}, {"scale", "SCALE"}, {"fakesirtiterations", "fake-sirt"},
      {"xtiltfile", "xtilt-file"}, {"zfactorfile", "zfactor-file"}, {"localfile", "local-file"},
      {"hamming", "hamming"}, {"exactfiltersize", "exact-filter-size"}};
  const std::vector<std::string> flags = {"gpu", "no-weight", "no-cosine-stretch", "log", "hamming",
                                          "exact-xtilt"};
  for (int i = 1; i < argc; ++i) {
    std::string arg = argv[i], val;
    bool has_eq = false;
    if (arg == "-h" || arg == "--help") { usage(stdout); exit(0); }
    std::string name;
    if (arg.rfind("--", 0) == 0) {
      size_t eq = arg.find('=');
      if (eq != std::string::npos) { val = arg.substr(eq + 1); arg = arg.substr(0, eq); has_eq = true; }
      auto it = alias.find(arg);
      name = it != alias.end() ? it->second : arg.substr(2);
    } else if (arg.size() == 2 && arg[0] == '-' && alias.count(arg)) {
      name = alias[arg];
    } else if (arg.size() > 2 && arg[0] == '-' && arg[1] != '-' && alias.count(arg.substr(0, 2)) &&
               !pip.count(lower(arg.substr(1)))) {
      name = alias[arg.substr(0, 2)];  // -z200 style
      val = arg.substr(2);
      has_eq = true;
    } else if (arg.size() > 1 && arg[0] == '-' && pip.count(lower(arg.substr(1)))) {
      name = pip[lower(arg.substr(1))];
    } else {
      clap_error("unexpected argument '" + arg + "' found");
    }
    bool is_flag = std::find(flags.begin(), flags.end(), name) != flags.end();
    if (name == "LOG") {  // PIP LOG takes a value (an offset); any value turns the log on
      if (i + 1 < argc && argv[i + 1][0] != '-') ++i;
      a.log = true;
      continue;
    }
    if (is_flag) {
      if (has_eq) clap_error("unexpected value '" + val + "' for '--" + name + "' found; no more were expected");
      if (name == "gpu") a.gpu = true;
      else if (name == "no-weight") a.no_weight = true;
      else if (name == "no-cosine-stretch") a.no_cosine_stretch = true;
      else if (name == "log") a.log = true;
      else if (name == "hamming") a.hamming = true;
      else if (name == "exact-xtilt") a.exact_xtilt = true;
      continue;
    }
    if (!has_eq) {
      if (i + 1 >= argc) clap_error("a value is required for '--" + name + "' but none was supplied");
      val = argv[++i];
    }
    if (name == "input") { a.input = val; has_in = true; }
    else if (name == "output") { a.output = val; has_out = true; }
    else if (name == "tilt-file") { a.tilt_file = val; has_tlt = true; }
    else if (name == "thickness") a.thickness = (int)parse_int(val, "--thickness", true);
    else if (name == "width") { a.width = (int)parse_int(val, "--width", true); a.has_width = true; }
    else if (name == "threads") a.threads = parse_int(val, "--threads", false);
    else if (name == "radial") a.radial = val;
    else if (name == "sirt") a.sirt = parse_int(val, "--sirt", false);
    else if (name == "sirt-relax") a.sirt_relax = parse_float(val, "--sirt-relax");
    else if (name == "local-file") a.local_file = val;
    else if (name == "xtilt-file") a.xtilt_file = val;
    else if (name == "zfactor-file") a.zfactor_file = val;
    else if (name == "densweight") a.densweight = parse_float(val, "--densweight");
    else if (name == "outscale") a.outscale = parse_float(val, "--outscale");
    else if (name == "outadd") a.outadd = parse_float(val, "--outadd");
    else if (name == "exact-filter-size") a.exact_filter_size = parse_int(val, "--exact-filter-size", false);
    else if (name == "fill-mode") a.fill_mode = val;
    else if (name == "cosine-interp") a.cosine_interp = val;
    else if (name == "max-cosine-tilt") a.max_cosine_tilt = parse_float(val, "--max-cosine-tilt");
    else if (name == "fake-sirt") a.fake_sirt = parse_int(val, "--fake-sirt", false);
    else if (name == "storage") a.storage = lower(val);
    else if (name == "device") a.device = (int)parse_int(val, "--device", false);
    else if (name == "io-chunk-kb") a.io_chunk_kb = std::max(1L, parse_int(val, "--io-chunk-kb", false));
    else if (name == "checkpoint") a.checkpoint = val;
    else if (name == "resume") a.resume = val;
    else if (name == "checkpoint-every") a.checkpoint_every = std::max(1L, parse_int(val, "--checkpoint-every", false));
    else if (name == "mode") {
      a.mode = (int)parse_int(val, "--mode", false);
      if (a.mode != 2 && a.mode != 12) clap_error("invalid value '" + val + "' for '--mode': 2 or 12");
    }
    else if (name == "SCALE") {  // IMOD: (v + add) * mult == (v * mult) + add*mult
      size_t c = val.find(',');
      float add = parse_float(val.substr(0, c), "-SCALE");
      float mult = c == std::string::npos ? 1.0f : parse_float(val.substr(c + 1), "-SCALE");
      a.outscale = mult;
      a.outadd = add * mult;
    } else clap_error("unexpected argument '--" + name + "' found");
  }
  std::string missing;
  if (!has_in) missing += "\n  --input <INPUT>";
  if (!has_out) missing += "\n  --output <OUTPUT>";
  if (!has_tlt) missing += "\n  --tilt-file <TILT_FILE>";
  if (!missing.empty()) clap_error("the following required arguments were not provided:" + missing);
  if ((!a.checkpoint.empty() || !a.resume.empty()) && (a.sirt <= 0 || a.gpu))
    clap_error("--checkpoint and --resume need SIRT iterations (--sirt > 0, without --gpu)");
  return a;
}

// First label of a checkpoint file: the iteration count and the run's total.
constexpr const char *CKPT_LABEL = "tiltgpu SIRT state: iterations ";
constexpr int CKPT_FILE_ERROR = 1;  // run_sirt_steps: a checkpoint file could not be read or written

// The raw SIRT volume ([y][out_nz][out_nx], before the output transform) as an
// MRC float volume of out_ny sections; written to FILE.tmp, then renamed, so an
// interrupted write leaves the previous checkpoint in place.
bool write_checkpoint(const std::string &path, const std::vector<float> &vol, int out_nx, int out_nz, int out_ny,
                      int done, int total, std::string *err) {
  mrc::Header h = mrc::Header::make(out_nx, out_nz, out_ny, mrc::FLOAT);
  h.add_label(std::string(CKPT_LABEL) + std::to_string(done) + " of " + std::to_string(total));
  const std::string tmp = path + ".tmp";
  {
    mrc::Writer w;
    if (!w.create(tmp, h, err)) return false;
    const size_t slice = (size_t)out_nx * out_nz;
    for (int y = 0; y < out_ny; ++y)
      if (!w.write_slice_f32(vol.data() + (size_t)y * slice, slice, err)) return false;
    if (!w.finish(0.0f, 0.0f, 0.0f, err)) return false;
  }
  if (std::rename(tmp.c_str(), path.c_str()) != 0) {
    *err = "cannot rename " + tmp + " to " + path;
    return false;
  }
  return true;
}

bool read_checkpoint(const std::string &path, std::vector<float> &vol, int out_nx, int out_nz, int out_ny,
                     int *done, std::string *err) {
  mrc::Reader r;
  if (!r.open(path, err)) return false;
  const mrc::Header &h = r.header();
  const std::string lab = h.nlabl > 0 ? h.label(0) : std::string();
  if (lab.rfind(CKPT_LABEL, 0) != 0) {
    *err = path + " is not a SIRT checkpoint of this program";
    return false;
  }
  *done = atoi(lab.c_str() + strlen(CKPT_LABEL));
  if (h.nx != out_nx || h.ny != out_nz || h.nz != out_ny || h.mode != mrc::FLOAT) {
    *err = path + ": volume size or mode does not match this reconstruction";
    return false;
  }
  vol.resize((size_t)out_nx * out_nz * out_ny);
  std::vector<float> sl;
  const size_t slice = (size_t)out_nx * out_nz;
  for (int y = 0; y < out_ny; ++y) {
    if (!r.read_slice_f32(y, sl, err) || sl.size() != slice) return false;
    std::copy(sl.begin(), sl.end(), vol.begin() + (size_t)y * slice);
  }
  return true;
}

// SIRT in steps (tg_sirt_*): from the WBP start or a --resume state, iterations in
// groups of --checkpoint-every, the state written after each group that leaves
// iterations to run, then the output stage.  Same volume as tg_reconstruct.
int run_sirt_steps(tg_session *s, const Args &args, int out_nx, int out_nz, int out_ny) {
  int rc, done = 0;
  const int total = (int)args.sirt;
  std::vector<float> vol;
  std::string err;
  if (!args.resume.empty()) {
    if (!read_checkpoint(args.resume, vol, out_nx, out_nz, out_ny, &done, &err)) {
      fprintf(stderr, "Error: %s\n", err.c_str());
      return CKPT_FILE_ERROR;
    }
    if ((rc = tg_sirt_restore(s, vol.data(), done)) != TG_OK) return rc;
    fprintf(stderr, "tilt: resuming SIRT after %d of %d iterations\n", done, total);
  } else if ((rc = tg_sirt_begin(s)) != TG_OK) {
    return rc;
  }
  const int every = args.checkpoint.empty() ? total : (int)args.checkpoint_every;
  while (done < total) {
    const int n = std::min(every, total - done);
    if ((rc = tg_sirt_iterate(s, n)) != TG_OK) return rc;
    done += n;
    if (!args.checkpoint.empty() && done < total) {
      vol.resize((size_t)out_nx * out_nz * out_ny);
      int32_t d = 0;
      if ((rc = tg_sirt_save(s, vol.data(), &d)) != TG_OK) return rc;
      if (!write_checkpoint(args.checkpoint, vol, out_nx, out_nz, out_ny, d, total, &err)) {
        fprintf(stderr, "Error: %s\n", err.c_str());
        return CKPT_FILE_ERROR;
      }
      fprintf(stderr, "tilt: SIRT state after %d of %d iterations written to %s\n", d, total,
              args.checkpoint.c_str());
    }
  }
  if ((rc = tg_sirt_end(s)) != TG_OK) return rc;
  return tg_synchronize(s);
}

}  // namespace

int main(int argc, char **argv) {
  Args args = parse(argc, argv);
  std::string err;
  std::vector<float> angles;
  if (!mrc::read_tilt_file(args.tilt_file, angles, &err)) {  // main.rs:550-553
    fprintf(stderr, "Error reading tilt file: %s\n", err.c_str());
    return 1;
  }
  mrc::Reader reader;
  if (!reader.open(args.input, &err)) {  // main.rs:555-558
    fprintf(stderr, "Error: %s\n", err.c_str());
    return 1;
  }
  const mrc::Header h = reader.header();
  const int in_nx = h.nx, in_ny = h.ny, nz = h.nz;
  const int out_nx = args.has_width ? args.width : h.nx;
  const int out_ny = in_ny;
  const int out_nz = args.thickness > 0 ? args.thickness : in_nx;
  fprintf(stderr, "tilt: %d projections, %d x %d -> %d x %d x %d (B200)\n", nz, in_nx, in_ny, out_nx,
          out_ny, out_nz);
  // --radial: silently fall back to the defaults on parse failure (main.rs:580-585)
  float cutoff = 0.35f, falloff = 0.05f;
  {
    std::vector<std::string> parts;
    size_t s = 0;
    while (true) {
      size_t c = args.radial.find(',', s);
      parts.push_back(args.radial.substr(s, c == std::string::npos ? std::string::npos : c - s));
      if (c == std::string::npos) break;
      s = c + 1;
    }
    auto tr = [](std::string x) {
      size_t a = 0, b = x.size();
      while (a < b && isspace((unsigned char)x[a])) ++a;
      while (b > a && isspace((unsigned char)x[b - 1])) --b;
      return x.substr(a, b - a);
    };
    float v;
    if (parts.size() > 0 && mrc::parse_f32(tr(parts[0]), v)) cutoff = v;
    if (parts.size() > 1 && mrc::parse_f32(tr(parts[1]), v)) falloff = v;
  }
  std::vector<float> local_rows, xtilt, zfac;
  if (!args.local_file.empty() && !mrc::load_local_rows(args.local_file, local_rows, &err)) {
    fprintf(stderr, "Error reading local alignment file: %s\n", err.c_str());
    return 1;
  }
  if (!args.xtilt_file.empty() && !mrc::load_per_view_file(args.xtilt_file, xtilt, &err)) {
    fprintf(stderr, "Error reading xtilt file: %s\n", err.c_str());
    return 1;
  }
  if (!args.zfactor_file.empty() && !mrc::load_per_view_file(args.zfactor_file, zfac, &err)) {
    fprintf(stderr, "Error reading zfactor file: %s\n", err.c_str());
    return 1;
  }
  tg_geometry g{};
  g.nx = in_nx;
  g.ny = in_ny;
  g.nz = nz;
  g.out_nx = out_nx;
  g.out_nz = out_nz;
  g.n_angles = (int)angles.size();
  g.angles = angles.data();
  if (!args.xtilt_file.empty()) { g.n_xtilt = (int)xtilt.size(); g.xtilt = xtilt.data(); }
  if (!args.zfactor_file.empty()) { g.n_zfactor = (int)zfac.size(); g.zfactor = zfac.data(); }
  if (!args.local_file.empty()) {
    g.has_local = 1;
    g.n_local = (int)(local_rows.size() / 5);
    g.local = local_rows.data();
  }
  tg_options o;
  tg_options_default(&o);
  o.radial_cutoff = cutoff;
  o.radial_falloff = falloff;
  o.hamming = args.hamming;
  o.exact_filter_size = (int)args.exact_filter_size;
  o.no_weight = args.no_weight;
  std::string fm = lower(args.fill_mode);
  o.fill_mode = fm == "zero" ? TG_FILL_ZERO : fm == "edge" ? TG_FILL_EDGE : TG_FILL_MEAN;
  o.no_cosine_stretch = args.no_cosine_stretch;
  o.cosine_cubic = lower(args.cosine_interp) == "cubic";
  o.max_cosine_tilt = args.max_cosine_tilt;
  o.log_transform = args.log;
  o.sirt_iters = (int)args.sirt;
  o.sirt_relax = args.sirt_relax;
  o.fake_sirt = (int)args.fake_sirt;
  o.densweight = args.densweight;
  o.outscale = args.outscale;
  o.outadd = args.outadd;
  o.gpu_compat = args.gpu;
  o.storage = args.storage == "fp16" ? TG_STORE_FP16 : args.storage == "bf16" ? TG_STORE_BF16 : TG_STORE_FP32;
  o.device = args.device;
  o.exact_xtilt = args.exact_xtilt;
  tg_session *s = nullptr;
  int rc = tg_session_create(&g, &o, &s);
  if (rc == TG_ERR_PANIC) {  // the reference indexes tilt_angles out of bounds and panics
    fprintf(stderr, "thread 'main' panicked: %s\n", tg_last_error());
    return 101;
  }
  if (rc != TG_OK) {
    fprintf(stderr, "Error: %s (%s)\n", tg_status_string(rc), tg_last_error());
    return 1;
  }
  auto fail = [&](int r) {
    fprintf(stderr, "Error: %s (%s)\n", tg_status_string(r), tg_last_error());
    tg_session_destroy(s);
    return 1;
  };
  using clk = std::chrono::steady_clock;
  auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
  const auto t_read0 = clk::now();
  // ---- input: a reader thread fills two pinned chunks of sections (read_slice_f32,
  // read.rs:127-231) while the previous chunk is copied to the device
  const size_t sec = (size_t)in_nx * in_ny;
  const size_t chunk_bytes = (size_t)args.io_chunk_kb << 10;
  const int zc = std::max(1, (int)std::min<size_t>((size_t)nz, chunk_bytes / (sec * 4)));
  void *pin_in[2] = {nullptr, nullptr};
  for (auto &p : pin_in)
    if ((rc = tg_host_alloc((size_t)zc * sec * 4, &p)) != TG_OK) return fail(rc);
  {
    std::mutex mu;
    std::condition_variable cv;
    int filled[2] = {-1, -1};  // chunk index held by each slot, -1: free
    bool read_failed = false, stop = false;  // stop: the uploader gave up, the reader quits
    std::string read_err;
    const int nchunks = (nz + zc - 1) / zc;
    std::thread rd([&] {
      std::vector<float> sl;
      std::string e;
      for (int k = 0; k < nchunks; ++k) {
        {
          std::unique_lock<std::mutex> lk(mu);
          cv.wait(lk, [&] { return filled[k % 2] < 0 || stop; });
          if (stop) return;
        }
        float *dst = static_cast<float *>(pin_in[k % 2]);
        const int z0 = k * zc, z1 = std::min(nz, z0 + zc);
        for (int z = z0; z < z1; ++z) {
          if (!reader.read_slice_f32(z, sl, &e) || sl.size() != sec) {
            std::lock_guard<std::mutex> lk(mu);
            read_failed = true;
            read_err = e.empty() ? "unsupported slice layout" : e;
            filled[k % 2] = k;
            cv.notify_all();
            return;
          }
          std::copy(sl.begin(), sl.end(), dst + (size_t)(z - z0) * sec);
        }
        std::lock_guard<std::mutex> lk(mu);
        filled[k % 2] = k;
        cv.notify_all();
      }
    });
    int up_rc = TG_OK;
    for (int k = 0; k < nchunks; ++k) {
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return filled[k % 2] == k; });
        if (read_failed) break;
      }
      const int z0 = k * zc, z1 = std::min(nz, z0 + zc);
      if ((up_rc = tg_upload_sections(s, z0, z1, static_cast<float *>(pin_in[k % 2]))) == TG_OK)
        up_rc = tg_synchronize(s);  // the slot may be refilled once its copy is done
      std::lock_guard<std::mutex> lk(mu);
      filled[k % 2] = -1;
      if (up_rc != TG_OK) stop = true;
      cv.notify_all();
      if (up_rc != TG_OK) break;
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      if (read_failed) stop = true;
      cv.notify_all();
    }
    rd.join();
    for (auto &p : pin_in) tg_host_free(p);
    if (up_rc != TG_OK) return fail(up_rc);
    if (read_failed) {
      fprintf(stderr, "Error: %s\n", read_err.c_str());
      tg_session_destroy(s);
      return 1;
    }
  }
  const auto t_rec0 = clk::now();
  const bool steps = args.sirt > 0 && !args.gpu && (!args.checkpoint.empty() || !args.resume.empty());
  if (!steps) {
    if ((rc = tg_reconstruct(s)) != TG_OK || (rc = tg_synchronize(s)) != TG_OK) return fail(rc);
  } else if ((rc = run_sirt_steps(s, args, out_nx, out_nz, out_ny)) != TG_OK) {
    if (rc == CKPT_FILE_ERROR) {  // reported already
      tg_session_destroy(s);
      return 1;
    }
    return fail(rc);
  }
  const auto t_rec1 = clk::now();
  uint8_t hin[1024], hout[1024];  // main.rs:710-717
  h.to_bytes(hin, false);
  tg_tilt_output_header(hin, out_nx, out_nz, hout);
  mrc::Header oh = mrc::Header::from_bytes(hout, false);
  if (args.mode == 12) oh.mode = mrc::HALF;
  mrc::Writer w;
  if (!w.create(args.output, oh, &err)) {
    fprintf(stderr, "Error: %s\n", err.c_str());
    tg_session_destroy(s);
    return 1;
  }
  // ---- output: chunk k+1 is copied off the device into one pinned buffer while
  // chunk k is written from the other (the reference writes each slice as it is
  // made, main.rs:1077-1085)
  const size_t slice = (size_t)out_nx * out_nz;
  const size_t eb = args.mode == 12 ? 2 : 4;
  const int chunk = std::max(1, (int)std::min<size_t>((size_t)out_ny, chunk_bytes / (slice * eb)));
  void *pin_out[2] = {nullptr, nullptr};
  for (auto &p : pin_out)
    if ((rc = tg_host_alloc((size_t)chunk * slice * eb, &p)) != TG_OK) return fail(rc);
  auto queue = [&](int y0, void *dst) {
    const int y1 = std::min(out_ny, y0 + chunk);
    return args.mode == 12 ? tg_download_slices_f16_async(s, y0, y1, static_cast<uint16_t *>(dst))
                           : tg_download_slices_async(s, y0, y1, static_cast<float *>(dst));
  };
  tg_stats st{};
  rc = tg_get_stats(s, &st);
  int k = 0;
  if (rc == TG_OK) rc = queue(0, pin_out[0]);
  for (int y0 = 0; rc == TG_OK && y0 < out_ny; y0 += chunk, ++k) {
    if ((rc = tg_synchronize(s)) != TG_OK) break;  // chunk k is in pin_out[k % 2]
    if (y0 + chunk < out_ny && (rc = queue(y0 + chunk, pin_out[(k + 1) % 2])) != TG_OK) break;
    const int y1 = std::min(out_ny, y0 + chunk);
    const uint8_t *src = static_cast<const uint8_t *>(pin_out[k % 2]);
    for (int y = y0; y < y1; ++y) {
      const bool ok = args.mode == 12 ? w.write_slice_raw(src + (size_t)(y - y0) * slice * 2, slice * 2, &err)
                                      : w.write_slice_f32(reinterpret_cast<const float *>(src) + (size_t)(y - y0) * slice,
                                                          slice, &err);
      if (!ok) {
        fprintf(stderr, "Error: %s\n", err.c_str());
        tg_synchronize(s);
        for (auto &p : pin_out) tg_host_free(p);
        tg_session_destroy(s);
        return 1;
      }
    }
    fprintf(stderr, "  %d/%d rows\n", y1, out_ny);
  }
  if (rc != TG_OK) {
    tg_synchronize(s);
    for (auto &p : pin_out) tg_host_free(p);
    return fail(rc);
  }
  for (auto &p : pin_out) tg_host_free(p);
  const auto t_wr1 = clk::now();
  fprintf(stderr, "tilt: read+upload %.3f s, reconstruct %.3f s, download+write %.3f s\n", secs(t_read0, t_rec0),
          secs(t_rec0, t_rec1), secs(t_rec1, t_wr1));
  tg_run_info info{};
  tg_session_last_run(s, &info);
  tg_session_destroy(s);
  if (!w.finish(st.amin, st.amax, st.amean, &err)) {
    fprintf(stderr, "Error: %s\n", err.c_str());
    return 1;
  }
  fprintf(stderr, "tilt: reconstruction complete -> %s (%.3f ms on GPU, %.3g voxel-view updates/s)\n",
          args.output.c_str(), info.ms_total, info.ms_total > 0 ? info.updates / (info.ms_total * 1e-3) : 0.0);
  return 0;
}
