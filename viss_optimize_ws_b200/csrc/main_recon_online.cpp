// Drop-in replacement of the upstream main_recon_online executable (and, built
// with VB_DEFAULTS_VISSFAST, of main_recon_online_mirror_tile_vissfast): same
// --key=value flags with prefix matching and silent fallback to the default
// on a parse error, same stdout lines, same output files
// (C{day}day{btag}.txt|.bin, Viss{day}day{btag}.txt, uvw/xyza/xyzb{day}day{btag}.txt).
// Upstream: main_recon_online.cu:5-586, common.hpp:58-153,
// mirror_tile_vissfast/main_recon_online_mirror_tile_vissfast.cu:6-709.
//
// All segments of a day run as one batch on one GPU (stage 1 and stage 2 each a
// persistent launch, replayed from a CUDA graph); the per-segment lines report
// each segment's share of the batched stage times.
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <mutex>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "vissb200.h"
#include "vb_text.h"

#if !defined(VB_DEFAULTS_ROOT) && !defined(VB_DEFAULTS_VISSFAST)
#define VB_DEFAULTS_ROOT 1
#endif

namespace {

struct Timer {
  std::chrono::high_resolution_clock::time_point t0;
  void tic() { t0 = std::chrono::high_resolution_clock::now(); }
  double toc_s() const {
    return std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
  }
};

// --key=value lookup, first match wins (common.hpp:58-64 semantics).
std::string get_arg(int argc, char** argv, const std::string& key, const std::string& defv) {
  for (int i = 1; i < argc; i++) {
    std::string s(argv[i]);
    if (s.rfind(key + "=", 0) == 0) return s.substr(key.size() + 1);
  }
  return defv;
}
int to_int(const std::string& s, int defv) { try { return std::stoi(s); } catch (...) { return defv; } }
double to_double(const std::string& s, double defv) { try { return std::stod(s); } catch (...) { return defv; } }
uint64_t to_u64(const std::string& s, uint64_t defv) { try { return (uint64_t)std::stoull(s); } catch (...) { return defv; } }

std::string norm_dir(std::string p) {
  while (!p.empty() && p.back() == '/') p.pop_back();
  return p;
}

int mkdir_p(const std::string& path) {
  std::string cur;
  std::stringstream ss(path);
  std::string part;
  if (!path.empty() && path[0] == '/') cur = "/";
  while (std::getline(ss, part, '/')) {
    if (part.empty()) continue;
    cur += part + "/";
    mkdir(cur.c_str(), 0755);
  }
  return 0;
}

// Sky loaders (common.hpp:89-143): text files may start with an npix header line.
bool load_txt(const std::string& path, float* out, long long n) {
  FILE* fp = fopen(path.c_str(), "r");
  if (!fp) return false;
  char line[256];
  if (!fgets(line, sizeof(line), fp)) { fclose(fp); return false; }
  char* p = line;
  float first = strtof(p, &p);
  long long i = 0;
  long long maybe = llround((double)first);
  if (!(std::llabs(maybe - n) == 0)) out[i++] = first;
  while (i < n && fgets(line, sizeof(line), fp)) {
    char* q = line;
    out[i++] = strtof(q, &q);
  }
  fclose(fp);
  return i == n;
}

bool load_bin(const std::string& path, float* out, long long n) {
  std::ifstream ifs(path, std::ios::binary);
  if (!ifs.is_open()) return false;
  ifs.read(reinterpret_cast<char*>(out), (std::streamsize)(n * (long long)sizeof(float)));
  return ifs.gcount() == (std::streamsize)(n * (long long)sizeof(float));
}

bool load_B_auto(const std::string& dir, const std::string& btag, float* out, long long npix,
                 const std::string& mode, std::string* used) {
  auto tt = [&](const std::string& p) { if (load_txt(p, out, npix)) { *used = p; return true; } return false; };
  auto tb = [&](const std::string& p) { if (load_bin(p, out, npix)) { *used = p; return true; } return false; };
  const std::string b1 = dir + "/B_" + btag + ".bin", b2 = dir + "/B.bin";
  const std::string t1 = dir + "/B_" + btag + ".txt", t2 = dir + "/B.txt";
  if (mode == "bin") return tb(b1) || tb(b2);
  if (mode == "txt") return tt(t1) || tt(t2);
  return tb(b1) || tb(b2) || tt(t1) || tt(t2);
}

// Failed writes are reported on stderr when the writer is drained.
std::string write_error(const std::string& path) { return "ERROR writing " + path + "\n"; }

struct Dev {
  vb_pipeline* p;
  std::vector<float> get(const char* name) {
    void* ptr = nullptr;
    int64_t n = 0;
    if (vb_pipeline_device_ptr(p, name, &ptr, &n) != VB_OK || !ptr || n <= 0) return {};
    std::vector<float> h((size_t)n);
    vb_memcpy(h.data(), ptr, (size_t)n * sizeof(float), VB_D2H);
    return h;
  }
};

int die(const std::string& msg) {
  std::cerr << msg << "\n";
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
#if defined(VB_DEFAULTS_VISSFAST)
  const bool vissfast = true;
#else
  const bool vissfast = false;
#endif
  std::string btag = get_arg(argc, argv, "--btag", "10M");
  int nside = to_int(get_arg(argc, argv, "--nside", "4096"), 4096);
  int day = to_int(get_arg(argc, argv, "--day", "1"), 1);
  int day_start = to_int(get_arg(argc, argv, "--day_start", std::to_string(day)), day);
  int day_count = vissfast ? to_int(get_arg(argc, argv, "--day_count", "1"), 1) : 1;
  if (!vissfast) day_start = day;
  int segs = to_int(get_arg(argc, argv, "--segs", "0"), 0);
  int blockage = to_int(get_arg(argc, argv, "--blockage", "1"), 1);
  int occ_mode = to_int(get_arg(argc, argv, "--occ_mode", "2"), 2);
  // upstream quirk: the root variant falls back to 1 on a parse error, the mirror variants to 0
  int write_viss = to_int(get_arg(argc, argv, "--write_viss", "0"), vissfast ? 0 : 1);
  int write_baseline_txt = to_int(get_arg(argc, argv, "--write_baseline_txt", "0"), 0);
  std::string B_mode = get_arg(argc, argv, "--B_mode", "auto");
  std::string C_mode = vissfast ? get_arg(argc, argv, "--C_mode", "bin") : get_arg(argc, argv, "--C_mode", "txt");
  int gen_gpu_index = to_int(get_arg(argc, argv, "--gen_gpu_index", "0"), 0);
  uint64_t orbit_seed = to_u64(get_arg(argc, argv, "--orbit_seed", "42"), 12345ULL);
  std::string sky_dir = norm_dir(get_arg(argc, argv, "--sky_dir", ""));
  std::string out_dir = get_arg(argc, argv, "--out_dir", "./out/");
  std::string gpus_s = get_arg(argc, argv, "--gpus", "0");
  if (!gpus_s.empty()) setenv("CUDA_VISIBLE_DEVICES", gpus_s.c_str(), 1);
  int print_stats = to_int(get_arg(argc, argv, "--print_stats", "1"), 1);
  int viss_tile_pix = to_int(get_arg(argc, argv, "--viss_tile_pix", "256"), 256);
  if (vissfast && viss_tile_pix != 256 && viss_tile_pix != 512 && get_arg(argc, argv, "--tile_any", "0") != "1")
    return die("ERROR --viss_tile_pix supports 256 or 512");

  // additive flags (this build)
  int mirror = to_int(get_arg(argc, argv, "--mirror", vissfast ? "1" : "0"), vissfast ? 1 : 0);
  int tilecone = to_int(get_arg(argc, argv, "--tilecone", vissfast ? "1" : "0"), vissfast ? 1 : 0);
  // 1: tiles the cone test proves visible skip the per-pixel test (the upstream
  // all-visible nm1 fast path); 0: they take it, only hidden tiles are culled
  int nm1_fast = to_int(get_arg(argc, argv, "--nm1_fast", "1"), 1);
  // exact sub-tiles inside tile-cone mixed tiles: 0 = default (128 pixels), < 0 = off
  int refine_pix = to_int(get_arg(argc, argv, "--refine_pix", "0"), 0);
  std::string prec_s = get_arg(argc, argv, "--precision", "fp32_fp64phase");
  std::string orbit_model = get_arg(argc, argv, "--orbit_model", "reference");
  int nsat = to_int(get_arg(argc, argv, "--nsat", "8"), 8);
  int tsteps = to_int(get_arg(argc, argv, "--tsteps", "0"), 0);
  double dt_s = to_double(get_arg(argc, argv, "--dt_s", "2"), 2.0);
  double alt_min = to_double(get_arg(argc, argv, "--alt_min_km", "400"), 400.0);
  double alt_max = to_double(get_arg(argc, argv, "--alt_max_km", "600"), 600.0);
  double spread = to_double(get_arg(argc, argv, "--spread_km", "50"), 50.0);
  double occ_R_m = to_double(get_arg(argc, argv, "--occ_R_m", "0"), 0.0);
  int grid_res = to_int(get_arg(argc, argv, "--grid_res", "0"), 0);
  double bl_max_m = to_double(get_arg(argc, argv, "--bl_max_m", "100000"), 100e3);
  std::string seg_plan = get_arg(argc, argv, "--seg_plan", "even");
  int seg_min = to_int(get_arg(argc, argv, "--seg_min_half", "50"), 50);
  int seg_max = to_int(get_arg(argc, argv, "--seg_max_half", "2000"), 2000);
  uint64_t seg_seed = to_u64(get_arg(argc, argv, "--seg_seed", "7"), 7);
  long long sky_gen = (long long)to_u64(get_arg(argc, argv, "--sky_gen", "0"), 0);
  int use_graph = to_int(get_arg(argc, argv, "--graph", "1"), 1);
  std::string report_json = get_arg(argc, argv, "--report_json", "");
  int stage2_cull = to_int(get_arg(argc, argv, "--stage2_cull", "2"), 2);
  int autotune = to_int(get_arg(argc, argv, "--autotune", "0"), 0);
  // cross-day running sum of the daily C (the upstream accumulator daemon,
  // viss_monitor.py / combine.py), kept on the device in FP64
  std::string accum_file = get_arg(argc, argv, "--accum_file", "");
  int keep_daily = to_int(get_arg(argc, argv, "--keep_daily", "1"), 1);
  // write each day's files on a background thread while the next day computes
  int async_write = to_int(get_arg(argc, argv, "--async_write", "1"), 1);
  // stream the sky through the device in slabs of this many pixels (0: resident)
  long long slab_pix = (long long)to_u64(get_arg(argc, argv, "--slab_pix", "0"), 0);

  if (btag != "1M" && btag != "10M" && btag != "30M") return die("ERROR --btag");
  if (nside <= 0) nside = (btag == "1M") ? 512 : (btag == "10M" ? 4096 : 16384);
  if (segs <= 0) segs = (btag == "1M") ? 1 : (btag == "10M" ? 10 : 30);
  if (sky_dir.empty()) sky_dir = (btag == "1M") ? "./earth_1Mhz" : (btag == "10M" ? "./earth_10Mhz" : "./earth_30Mhz");
  if (!out_dir.empty() && out_dir.back() != '/') out_dir.push_back('/');
  mkdir_p(out_dir);

  int precision = VB_PREC_FP32_FP64PH;
  if (prec_s == "fp64") precision = VB_PREC_FP64;
  else if (prec_s == "fp32_dsphase") precision = VB_PREC_FP32_DSPH;
  else if (prec_s == "ref32") precision = VB_PREC_REF32;
  else if (prec_s != "fp32_fp64phase") return die("ERROR --precision (fp64|fp32_fp64phase|fp32_dsphase|ref32)");
  int model = (orbit_model == "synthetic") ? VB_ORBIT_SYNTHETIC : VB_ORBIT_REFERENCE;
  if (orbit_model != "synthetic" && orbit_model != "reference") return die("ERROR --orbit_model (reference|synthetic)");

  int sm = 0, ccM = 0, ccm = 0;
  if (vb_device_info(&sm, &ccM, &ccm) != VB_OK)
    return die("ERROR no visible CUDA devices after applying CUDA_VISIBLE_DEVICES=" + gpus_s);
  const int G = 1;
  std::cout << "CUDA_VISIBLE_DEVICES=" << gpus_s << "\n";
  std::cout << "Visible logical GPUs: 0\n";
  long long npix = 12LL * nside * nside;
  if (vissfast)
    std::cout << "btag=" << btag << " nside=" << nside << " npix=" << npix << " day_start=" << day_start
              << " day_count=" << day_count << " segs=" << segs << "\n";
  else
    std::cout << "btag=" << btag << " nside=" << nside << " npix=" << npix << " day=" << day << " segs=" << segs
              << "\n";
  std::cout << "blockage=" << blockage << " occ_mode=" << occ_mode << "  [Viss stage: blockage=ON, phase_correct=ON]\n";
  std::cout << " sky_dir=" << sky_dir << " out_dir=" << out_dir << " gpus=" << gpus_s
            << (vissfast ? " C_mode=" + C_mode : std::string()) << "\n";

  float R = 1737.1e3f, h = 300e3f;
  float theta = asinf(R / (R + h));
  float phi = (float)M_PI - theta;
  float cosphi = cosf(phi);
  float frequency = (btag == "1M") ? 1e6f : (btag == "10M" ? 1e7f : 3e7f);
  float lamda = 3e8f / frequency;
  std::cout << "theta=" << theta << " phi=" << phi << " cosphi=" << cosphi << " lamda=" << lamda << "\n";

  // sky: optional seeded synthetic file in the upstream binary format
  if (sky_gen > 0) {
    std::vector<float> Bgen((size_t)npix);
    if (vb_make_synthetic_sky(nside, (uint64_t)sky_gen, 20, 10.0f, Bgen.data()) != VB_OK) return die(vb_last_error());
    mkdir_p(sky_dir);
    std::ofstream o(sky_dir + "/B_" + btag + ".bin", std::ios::binary);
    o.write(reinterpret_cast<const char*>(Bgen.data()), (std::streamsize)(npix * sizeof(float)));
    if (!o) return die("ERROR writing synthetic sky to " + sky_dir);
  }
  Timer t_io;
  t_io.tic();
  std::vector<float> hB((size_t)npix);
  std::string used;
  if (!load_B_auto(sky_dir, btag, hB.data(), npix, B_mode, &used))
    return die("ERROR reading B in mode=" + B_mode + " from " + sky_dir);
  std::cout << "Loaded B from " << used << " in " << t_io.toc_s() << " s\n";
  const double pix_area = 4.0 * M_PI / (double)npix;
  std::cout << " pix_area=" << pix_area << " inv_pix_area=" << (1.0 / pix_area) << "\n";

  if (gen_gpu_index < 0 || gen_gpu_index >= G)
    return die("ERROR gen_gpu_index out of range: " + std::to_string(gen_gpu_index) + " / " + std::to_string(G) +
               " (visible GPUs)");

  vb_run_config cfg;
  vb_run_config_defaults(&cfg);
  cfg.nside = nside;
  cfg.segs = segs;
  cfg.blockage = blockage;
  cfg.occ_mode = occ_mode;
  cfg.orbit_seed = orbit_seed;
  cfg.lambda_m = lamda;
  cfg.viss_tile_pix = viss_tile_pix;
  cfg.mirror = mirror;
  cfg.cull = tilecone ? VB_CULL_TILECONE : VB_CULL_EXACT;
  cfg.precision = precision;
  cfg.orbit_model = model;
  cfg.nsat = nsat;
  cfg.tsteps = tsteps;
  cfg.dt_s = dt_s;
  cfg.alt_min_km = alt_min;
  cfg.alt_max_km = alt_max;
  cfg.spread_km = spread;
  cfg.occ_R_m = occ_R_m;
  cfg.bl_max_m = (float)bl_max_m;
  cfg.grid_res = grid_res;
  cfg.seg_plan = (seg_plan == "uneven") ? 1 : 0;
  cfg.seg_min_half = seg_min;
  cfg.seg_max_half = seg_max;
  cfg.seg_seed = seg_seed;
  cfg.stage2_cull = stage2_cull;
  cfg.nm1_fast = nm1_fast ? 1 : 0;
  cfg.stage1_refine_pix = refine_pix;
  cfg.slab_pix = slab_pix;
  cfg.use_graph = use_graph;
  cfg.device = 0;

  // --report_json: the SFU (sin + cos) rate of this GPU, measured once, is the
  // denominator of the per-stage roofline fractions of each day
  double sfu_pairs = 0.0;
  if (!report_json.empty()) {
    double f32 = 0, f64 = 0, clk = 0;
    if (vb_measure_peaks(&sfu_pairs, &f32, &f64, &clk) != VB_OK) sfu_pairs = 0.0;
  }
  std::ostringstream json;
  json << "{\"sfu_pairs_per_s\": " << sfu_pairs << ", \"days\": [";
  // one run context for all days: each further day only swaps the orbit
  vbtext::AsyncWriter writer(async_write != 0);
  vb_pipeline* p = nullptr;
  double* d_acc = nullptr;
  for (int di = 0; di < day_count; ++di) {
    const int dayid = day_start + di;
    cfg.day = dayid;
    writer.drain(std::cout);
    if (vissfast) std::cout << "===== Day " << dayid << " / " << (day_start + day_count - 1) << " =====\n";
    Timer t_init;
    t_init.tic();
    if (!p) {
      int rc = vb_pipeline_create(&cfg, &p);
      if (rc == VB_ERR_NOMEM && !slab_pix) {
        // The sky does not fit on the device with its stage-1 records (the
        // upstream's 30 MHz sky, nside 16384, needs ~320 GB resident): stream
        // it through in slabs of whole cull tiles and stage-2 pixel blocks, a
        // power of two half the largest that fits, so that the running sum
        // and the rest of the run keep room on the device.
        const long long unit = std::max<long long>(1024, cfg.viss_tile_pix > 0 ? cfg.viss_tile_pix : 256);
        long long s = 1;
        while (s * 2 <= npix / 2) s *= 2;
        for (; s >= unit && rc == VB_ERR_NOMEM; s /= 2) {
          cfg.slab_pix = s;
          rc = vb_pipeline_create(&cfg, &p);
          if (rc == VB_OK) slab_pix = s;
        }
        if (rc == VB_OK && slab_pix / 2 >= unit) {
          vb_pipeline_destroy(p);
          p = nullptr;
          cfg.slab_pix = slab_pix / 2;
          rc = vb_pipeline_create(&cfg, &p);
          if (rc == VB_OK) slab_pix = cfg.slab_pix;
        }
        if (rc == VB_OK)
          std::cout << "Sky of " << npix << " pixels does not fit on the device: streaming it in slabs of "
                    << slab_pix << " pixels\n";
      }
      if (rc != VB_OK) return die(std::string("ERROR ") + vb_last_error());
      if (!slab_pix && vb_pipeline_set_sky(p, hB.data(), 1) != VB_OK)
        return die(std::string("ERROR ") + vb_last_error());
      if (!accum_file.empty()) {
        // resume from an existing running sum (float32, npix) or start at zero
        if (vb_malloc(reinterpret_cast<void**>(&d_acc), (size_t)npix * sizeof(double)) != VB_OK)
          return die(std::string("ERROR ") + vb_last_error());
        std::vector<double> a((size_t)npix, 0.0);
        std::ifstream in(accum_file, std::ios::binary | std::ios::ate);
        if (in.is_open()) {
          if ((int64_t)in.tellg() != npix * (int64_t)sizeof(float))
            return die("ERROR accum_file " + accum_file + " does not hold npix float32 values");
          in.seekg(0);
          std::vector<float> f((size_t)npix);
          in.read(reinterpret_cast<char*>(f.data()), (std::streamsize)(npix * sizeof(float)));
          if (!in) return die("ERROR reading " + accum_file);
          for (int64_t i = 0; i < npix; ++i) a[i] = f[i];
          std::cout << "Resuming running sum from " << accum_file << "\n";
        }
        if (vb_memcpy(d_acc, a.data(), a.size() * sizeof(double), VB_H2D) != VB_OK)
          return die(std::string("ERROR ") + vb_last_error());
      }
    } else if (vb_pipeline_set_day(p, dayid) != VB_OK) {
      return die(std::string("ERROR ") + vb_last_error());
    }
    int64_t np_ = 0;
    int nseg = 0, n_half = 0, nbl = 0, ntile = 0;
    float cp = 0;
    vb_pipeline_info(p, &np_, &nseg, &n_half, &nbl, &ntile, &cp);
    std::vector<int> t0(nseg), tl(nseg);
    vb_pipeline_seg_plan(p, t0.data(), tl.data());
    int max_tlen = *std::max_element(tl.begin(), tl.end());
    if (di == 0) {
      int orr = 0, pc = 0, sl = 0;
      if (model == VB_ORBIT_REFERENCE) {
        vb_orbit_params op{};
        op.model = VB_ORBIT_REFERENCE;
        op.lambda_m = lamda;
        op.day = dayid;
        op.seed = orbit_seed;
        op.nsat = 8;
        vb_orbit* o = nullptr;
        int T = 0;
        if (vb_orbit_create(&op, &o) == VB_OK) {
          vb_orbit_info(o, &T, nullptr, &orr, &pc, &sl);
          vb_orbit_destroy(o);
        }
      }
      long long Tsum = 0;
      for (int k = 0; k < nseg; ++k) Tsum += tl[k];
      std::cout << "Online orbit plan: OrbitRes=" << orr << " ProcessionCount=" << pc << " segLen=" << sl
                << " T=" << Tsum << " N=" << Tsum * 2 * nbl << "\n";
      std::cout << "Segment plan: max_tlen=" << max_tlen << " max_segN=" << (long long)max_tlen * 2 * nbl
                << " max_segN_half=" << (long long)max_tlen * nbl << "\n";
    }
    int rc = vb_pipeline_make_baselines(p);
    if (rc == VB_ERR_HALFSYM) return die(std::string("ERROR: generated segment uvw does not satisfy half-sym: ") + vb_last_error());
    if (rc != VB_OK) return die(std::string("ERROR ") + vb_last_error());
    if (autotune && di == 0 && slab_pix) std::cout << "Autotune skipped: not available in sky-slab mode\n";
    if (autotune && di == 0 && !slab_pix) {
      // kernel shapes for this workload, kept for the following days
      vb_tune_report tr{};
      if (vb_pipeline_autotune(p, 2, &tr) != VB_OK) return die(std::string("ERROR autotune: ") + vb_last_error());
      cfg.stage1_bpt = tr.stage1_bpt;
      cfg.stage1_stage_pix = tr.stage1_stage_pix;
      cfg.stage1_ctas_per_sm = tr.stage1_ctas_per_sm;
      cfg.stage1_items_per_cta = tr.stage1_items_per_cta;
      cfg.stage2_ppt = tr.stage2_ppt;
      cfg.stage2_items_per_cta = tr.stage2_items_per_cta;
      std::cout << "Autotune: stage1 bpt=" << tr.stage1_bpt << " stage_pix=" << tr.stage1_stage_pix
                << " ctas_per_sm=" << tr.stage1_ctas_per_sm << " items_per_cta=" << tr.stage1_items_per_cta << " "
                << tr.stage1_ms << " ms (auto " << tr.stage1_default_ms << " ms); stage2 ppt=" << tr.stage2_ppt
                << " items_per_cta=" << tr.stage2_items_per_cta << " " << tr.stage2_ms << " ms (auto "
                << tr.stage2_default_ms << " ms); " << tr.candidates << " shapes timed\n";
    }
    std::cout << "Init GPUs in " << t_init.toc_s() << " s\n";
    std::cout << "Orbit generator initialized on dev=0\n";
    std::cout << "Baseline broadcast: gen_dev=0 need_host_stage=0\n";

    Timer t_rec;
    t_rec.tic();
    vb_report rep;
    std::vector<float> Cslab;
    if (slab_pix) {
      // sky-slab mode: B streams from host memory, C comes back slab by slab
      Cslab.resize((size_t)npix);
      if (vb_pipeline_run_host(p, hB.data(), 1, Cslab.data(), nullptr, &rep) != VB_OK)
        return die(std::string("ERROR ") + vb_last_error());
    } else if (vb_pipeline_run(p, &rep) != VB_OK) {
      return die(std::string("ERROR ") + vb_last_error());
    }
    if (rep.error_flags != 0)   // stderr only: stdout keeps the upstream lines
      std::cerr << "WARNING day " << dayid << ": device error flags " << rep.error_flags
                << ((rep.error_flags & VB_DEVERR_PHASE_RANGE) ? " (uvw beyond the fp32_fp64phase range; use --precision=fp64)" : "")
                << ": this day's outputs are not to be trusted" << std::endl;
    std::vector<vb_seg_params> sp(nseg);
    vb_pipeline_seg_params(p, sp.data());
    Dev dv{p};
    std::vector<float> hu, hv, hw;
    if (print_stats || write_baseline_txt) { hu = dv.get("u"); hv = dv.get("v"); hw = dv.get("w"); }
    const std::string dtag = std::to_string(dayid) + "day" + btag;
    if (write_viss) {
      // "re im" per signed baseline, printf %g as the upstream iostream output
      std::string fv = out_dir + "Viss" + dtag + ".txt";
      std::cout << "Will stream phase-corrected Viss to " << fv << "\n";
      auto Vf = std::make_shared<std::vector<float>>(dv.get("V_full"));
      writer.submit([&writer, fv, Vf] {
        const bool ok = vbtext::write_rows(fv, {{Vf->data(), 2}, {Vf->data() + 1, 2}}, Vf->size() / 2,
                                           vbtext::Fmt::General6);
        if (!ok) writer.log(write_error(fv));
        return ok;
      });
    }
    if (write_baseline_txt) {
      std::cout << "Will stream generated uvw/xyza/xyzb to txt under " << out_dir << "\n";
      auto tab = std::make_shared<std::vector<std::vector<float>>>();
      tab->push_back(hu);
      tab->push_back(hv);
      tab->push_back(hw);
      for (const char* k : {"x1", "y1", "z1", "x2", "y2", "z2"}) tab->push_back(dv.get(k));
      const std::string names[3] = {out_dir + "uvw" + dtag + ".txt", out_dir + "xyza" + dtag + ".txt",
                                    out_dir + "xyzb" + dtag + ".txt"};
      for (int f = 0; f < 3; ++f) {
        const std::string fn = names[f];
        writer.submit([&writer, fn, tab, f] {
          const auto& t = *tab;
          const bool ok = vbtext::write_rows(fn, {{t[3 * f].data(), 1}, {t[3 * f + 1].data(), 1}, {t[3 * f + 2].data(), 1}},
                                             t[3 * f].size(), vbtext::Fmt::Sci15);
          if (!ok) writer.log(write_error(fn));
          return ok;
        });
      }
    }
    // per-segment lines: each segment's share of the batched stage times
    const double tot_s1 = (double)rep.n_half_total;
    const double tot_s2 = (double)std::max<long long>(1, rep.groups_total);
    for (int s = 0; s < nseg; ++s) {
      const int segN = tl[s] * 2 * nbl, segNh = tl[s] * nbl;
      const double tv = rep.t_stage1_ms * 1e-3 * segNh / tot_s1;
      const double tr = rep.t_stage2_ms * 1e-3 * sp[s].nuniq / tot_s2;
      if (sp[s].nuniq <= 0) {
        std::cout << (vissfast ? "[day " + std::to_string(dayid) + " seg " : std::string("[seg ")) << (s + 1) << "/"
                  << nseg << "] nuniq<=0, skip\n";
        continue;
      }
      std::ostringstream line;
      if (vissfast) line << "[day " << dayid << " seg " << (s + 1) << "/" << nseg << "]";
      else line << "[seg " << (s + 1) << "/" << nseg << "]";
      line << " t0=" << t0[s] << " segN=" << segN << " segN_half=" << segNh << " VissTime=" << tv << "s"
           << " ReconSegTime=" << tr << "s" << " fa=" << sp[s].fa << " fb=" << sp[s].fb << " denom=" << sp[s].denom
           << (vissfast ? " nuniq_halfgrid=" : " nuniq=") << sp[s].nuniq << " RES=" << sp[s].RES;
      if (print_stats && !hu.empty()) {
        const int i0 = t0[s] * 2 * nbl;
        float umin = INFINITY, umax = -INFINITY, vmin = INFINITY, vmax = -INFINITY, wmin = INFINITY, wmax = -INFINITY;
        for (int i = i0; i < i0 + segN; ++i) {
          umin = std::min(umin, hu[i]); umax = std::max(umax, hu[i]);
          vmin = std::min(vmin, hv[i]); vmax = std::max(vmax, hv[i]);
          wmin = std::min(wmin, hw[i]); wmax = std::max(wmax, hw[i]);
        }
        line << " u=[" << umin << "," << umax << "] v=[" << vmin << "," << vmax << "] w=[" << wmin << "," << wmax
             << "]";
      }
      std::cout << line.str() << "\n";
    }
    std::cout << "Recon done in " << t_rec.toc_s() << " s\n";

    std::vector<float> Cout = slab_pix ? std::move(Cslab) : dv.get("C");
    const bool txt = (C_mode == "txt");
    std::string outC = out_dir + "C" + dtag + (txt ? ".txt" : ".bin");
    if (d_acc) {
      // running sum: device FP64 += C, file = float32 sum, log line per day
      Timer t_a;
      t_a.tic();
      void* dC = nullptr;
      int64_t nC = 0;
      if (vb_pipeline_device_ptr(p, "C", &dC, &nC) != VB_OK) return die(std::string("ERROR ") + vb_last_error());
      if (slab_pix) {
        // the device holds one slab of C: add the host copy slab-sized piece by piece
        for (int64_t b0 = 0; b0 < npix; b0 += nC) {
          const int64_t cnt = std::min<int64_t>(nC, npix - b0);
          if (vb_memcpy(dC, Cout.data() + b0, (size_t)cnt * sizeof(float), VB_H2D) != VB_OK ||
              vb_accumulate(static_cast<const float*>(dC), cnt, d_acc + b0, nullptr) != VB_OK)
            return die(std::string("ERROR ") + vb_last_error());
        }
      } else if (vb_accumulate(static_cast<const float*>(dC), nC, d_acc, nullptr) != VB_OK) {
        return die(std::string("ERROR ") + vb_last_error());
      }
      if (vb_synchronize() != VB_OK) return die(std::string("ERROR ") + vb_last_error());
      std::vector<double> a((size_t)npix);
      if (vb_memcpy(a.data(), d_acc, a.size() * sizeof(double), VB_D2H) != VB_OK)
        return die(std::string("ERROR ") + vb_last_error());
      std::vector<float> f((size_t)npix);
      double mean = 0.0, mn = INFINITY, mx = -INFINITY;
      for (int64_t i = 0; i < npix; ++i) {
        f[i] = (float)a[i];
        mean += a[i];
        mn = std::min(mn, a[i]);
        mx = std::max(mx, a[i]);
      }
      mean /= (double)npix;
      std::ofstream o(accum_file, std::ios::binary | std::ios::trunc);
      o.write(reinterpret_cast<const char*>(f.data()), (std::streamsize)(npix * sizeof(float)));
      if (!o) return die("ERROR writing " + accum_file);
      o.close();
      std::time_t now = std::time(nullptr);
      char ts[32];
      std::strftime(ts, sizeof(ts), "%Y-%m-%d %H:%M:%S", std::localtime(&now));
      std::ofstream lg(accum_file + ".log", std::ios::app);
      lg << ts << " | C" << dayid << " | time=" << std::fixed << std::setprecision(1) << t_a.toc_s()
         << "s | mean=" << std::setprecision(6) << mean << "\n";
      std::cout << "Accumulated day " << dayid << " into " << accum_file << ": mean=" << mean << " min=" << mn
                << " max=" << mx << "\n";
    }
    if (!keep_daily) {
      std::cout << "Daily C not written (--keep_daily=0)\n";
    } else {
      auto Ch = std::make_shared<std::vector<float>>(std::move(Cout));
      writer.submit([&writer, outC, Ch, txt] {
        Timer tw;
        tw.tic();
        const bool ok = txt ? vbtext::write_rows(outC, {{Ch->data(), 1}}, Ch->size(), vbtext::Fmt::General6)
                            : vbtext::write_binary(outC, Ch->data(), Ch->size() * sizeof(float));
        if (!ok) {
          writer.log(write_error(outC));
          return false;
        }
        std::ostringstream m;
        m << "Wrote " << outC << " in " << tw.toc_s() << " s\n";
        writer.log(m.str());
        return true;
      });
    }
    json << (di ? ", " : "") << "{\"day\": " << dayid << ", \"t_stage1_ms\": " << rep.t_stage1_ms
         << ", \"t_stage2_ms\": " << rep.t_stage2_ms << ", \"stage1_terms\": " << rep.stage1_terms
         << ", \"stage2_terms\": " << rep.stage2_terms << ", \"groups\": " << rep.groups_total
         << ", \"error_flags\": " << rep.error_flags << ", \"t_s1_kernel_ms\": " << rep.t_s1_kernel_ms
         << ", \"t_s2_kernel_ms\": " << rep.t_s2_kernel_ms << ", \"s1_counters\": [" << rep.s1_counters[0] << ", "
         << rep.s1_counters[1] << ", " << rep.s1_counters[2] << ", " << rep.s1_counters[3]
         << "], \"s2_counters\": [" << rep.s2_counters[0] << ", " << rep.s2_counters[1] << ", "
         << rep.s2_counters[2] << ", " << rep.s2_counters[3] << "]";
    // evaluated terms (visible-fast + masked) per second over the kernel time, against the SFU rate
    auto frac = [&](const unsigned long long* c, double ms) {
      return (sfu_pairs > 0 && ms > 0) ? (double)(c[0] + c[1]) / (ms * 1e-3) / sfu_pairs : 0.0;
    };
    json << ", \"stage1_sfu_frac\": " << frac(rep.s1_counters, rep.t_s1_kernel_ms)
         << ", \"stage2_sfu_frac\": " << frac(rep.s2_counters, rep.t_s2_kernel_ms) << "}";
  }
  if (p) vb_pipeline_destroy(p);
  if (d_acc) vb_free(d_acc);
  const bool wrote = writer.wait();
  writer.drain(std::cout);
  if (!wrote) return die("ERROR writing outputs");
  json << "]}";
  if (!report_json.empty()) {
    std::ofstream o(report_json);
    o << json.str() << "\n";
  }
  return 0;
}
