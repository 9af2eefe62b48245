// Seeded synthetic input generator for the pixel reconstruction chain.
//
// It builds a Phase-1-like pixel geometry (4 barrel layers at r = 2.9/6.8/
// 10.9/16.0 cm, 3 forward disks per side at |z| = 32/39/48 cm, 1856 modules of
// 160x416 pixels, 100x150 um pitch, B = 3.8 T) and writes the conditions and the
// raw events in the reference's own on-disk layouts:
//   cablingMap.bin  SiPixelFedCablingMapGPUWrapperESProducer.jl:27-46
//   fedIds.bin      SiPixelFedCablingMapGPUWrapperESProducer.jl:50-57
//   gain.bin        SiPixelGainCalibrationForHLTGPUESProducer.jl:14-46
//   cpefast.bin     PixelCPEFastESProducer.jl:16-103
//   beamspot.bin    BeamSpotESProducer.jl:11-28
//   raw.bin         bin/ReadRAW.jl:9-31 (per event: i32 nFeds, then per FED
//                   i32 fedId, i32 size, size bytes)
// Events are helix tracks from one or more vertices, digitised into pixels with
// Landau-like charge and packed into FED words with the same bit layout that
// raw_to_digi_kernal decodes (SiPixelRawToClusterGPUKernel.jl:37-105, 537-658).
// This is input synthesis only: nothing here is on the reconstruction path.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <random>
#include <thread>
#include <vector>

namespace {

constexpr int kModules = 1856;
constexpr int kLadders = 148;
constexpr int kRows = 160, kCols = 416;
constexpr int kMaxFed = 150, kMaxLink = 48, kMaxRoc = 8;
constexpr int kCablingSize = kMaxFed * kMaxLink * kMaxRoc;  // 57600
constexpr int kFedBase = 1200;
constexpr int kModulesPerFed = 24;                          // 2 links per module
constexpr float kPitchX = 0.01f, kPitchY = 0.015f;
constexpr float kThickB = 0.0285f, kThickE = 0.029f;
constexpr double kBField = 3.8;
constexpr double kInvRadiusPerGeV = 0.0114256972711507;  // 1/(R[cm] * pT[GeV]) at 3.8 T
const int kLayerStart[11] = {0, 96, 320, 672, 1184, 1296, 1408, 1520, 1632, 1744, 1856};
const int kLaddersPerLayer[4] = {12, 28, 44, 64};
const double kBarrelR[4] = {2.9, 6.8, 10.9, 16.0};
const double kDiskZ[3] = {32.0, 39.0, 48.0};

struct Module {
  bool barrel;
  int layer;   // barrel 1..4, endcap disk 1..3
  int side;    // endcap: +1 / -1
  int ladder;  // barrel ladder index or endcap blade index
  int modz;    // barrel module 1..8 along z; endcap ring 0/1
  uint32_t raw_id;
  double p[3];
  double R[9];  // rows are the local x, y, z axes in global coordinates
  float x0, y0, z0;
};

struct Geometry {
  std::vector<Module> mods;
  Geometry() {
    mods.resize(kModules);
    for (int L = 0; L < 4; ++L) {
      int nl = kLaddersPerLayer[L];
      for (int k = 0; k < nl; ++k) {
        double phi = 2.0 * M_PI * (k + 0.25 * L) / nl;
        double r = kBarrelR[L] + ((k & 1) ? 0.15 : -0.15);
        for (int mz = 0; mz < 8; ++mz) {
          int id = kLayerStart[L] + k * 8 + mz;
          Module& m = mods[id];
          m.barrel = true; m.layer = L + 1; m.side = mz < 4 ? -1 : 1; m.ladder = k; m.modz = mz + 1;
          m.raw_id = (1u << 28) | (1u << 25) | (uint32_t(L + 1) << 20) | (uint32_t(k + 1) << 12) | (uint32_t(mz + 1) << 2);
          m.p[0] = r * std::cos(phi); m.p[1] = r * std::sin(phi); m.p[2] = (mz - 3.5) * 6.5;
          double ex[3] = {-std::sin(phi), std::cos(phi), 0}, ey[3] = {0, 0, 1}, ez[3] = {std::cos(phi), std::sin(phi), 0};
          for (int j = 0; j < 3; ++j) { m.R[j] = ex[j]; m.R[3 + j] = ey[j]; m.R[6 + j] = ez[j]; }
        }
      }
    }
    for (int s = 0; s < 2; ++s) {
      for (int d = 0; d < 3; ++d) {
        int base = kLayerStart[4 + 3 * s + d];
        double zd = (s == 0 ? 1.0 : -1.0) * kDiskZ[d];
        int idx = 0;
        for (int ring = 0; ring < 2; ++ring) {
          int n = ring == 0 ? 44 : 68;
          double rc = ring == 0 ? 7.0 : 13.0;
          for (int k = 0; k < n; ++k, ++idx) {
            double phi = 2.0 * M_PI * (k + 0.5 * ring) / n;
            Module& m = mods[base + idx];
            m.barrel = false; m.layer = d + 1; m.side = s == 0 ? 1 : -1; m.ladder = k; m.modz = ring;
            uint32_t side_bits = s == 0 ? 2u : 1u;
            m.raw_id = (1u << 28) | (2u << 25) | (side_bits << 23) | (uint32_t(d + 1) << 18) | (uint32_t(k + 1) << 12) |
                       (uint32_t(ring + 1) << 10) | (1u << 2);
            m.p[0] = rc * std::cos(phi); m.p[1] = rc * std::sin(phi); m.p[2] = zd + ((k & 1) ? 0.25 : -0.25);
            double ex[3] = {-std::sin(phi), std::cos(phi), 0}, ey[3] = {std::cos(phi), std::sin(phi), 0}, ez[3] = {0, 0, -1};
            for (int j = 0; j < 3; ++j) { m.R[j] = ex[j]; m.R[3 + j] = ey[j]; m.R[6 + j] = ez[j]; }
          }
        }
      }
    }
    for (auto& m : mods) {
      // local coordinates of the global origin: x0,y0,z0 in the CPE angle estimate
      double v[3] = {-m.p[0], -m.p[1], -m.p[2]};
      m.x0 = float(m.R[0] * v[0] + m.R[1] * v[1] + m.R[2] * v[2]);
      m.y0 = float(m.R[3] * v[0] + m.R[4] * v[1] + m.R[5] * v[2]);
      m.z0 = float(m.R[6] * v[0] + m.R[7] * v[1] + m.R[8] * v[2]);
    }
  }
};

const Geometry& geom() {
  static Geometry g;
  return g;
}

// ROC -> module pixel mapping, the frame conversion the unpacker applies
// (SiPixelRawToClusterGPUKernel.jl:271-350). The generator inverts it by table.
void roc_to_module(bool bpix, int side, int layer, int roc, int r, int c, int* row, int* col) {
  int sr, sc, ro, co;
  bool minus = bpix ? (side == -1 && layer != 1) : (side == -1);
  bool flip_first = bpix ? minus : true;  // fpix: both panels use the same mapping
  if (flip_first) {
    if (roc < 8) { sr = 1; sc = -1; ro = 0; co = (8 - roc) * 52 - 1; }
    else { sr = -1; sc = 1; ro = 2 * 80 - 1; co = (roc - 8) * 52; }
  } else {
    if (roc < 8) { sr = -1; sc = 1; ro = 2 * 80 - 1; co = roc * 52; }
    else { sr = 1; sc = -1; ro = 0; co = (16 - roc) * 52 - 1; }
  }
  *row = sr * r + ro;
  *col = sc * c + co;
}

struct InvMap {  // module (row,col) -> (roc, r, c) for one mapping flavour
  std::vector<uint16_t> roc, r, c;
  InvMap(bool bpix, int side, int layer) : roc(kRows * kCols), r(kRows * kCols), c(kRows * kCols) {
    for (int ro = 0; ro < 16; ++ro)
      for (int rr = 0; rr < 80; ++rr)
        for (int cc = 0; cc < 52; ++cc) {
          int row, col;
          roc_to_module(bpix, side, layer, ro, rr, cc, &row, &col);
          int k = row * kCols + col;
          roc[k] = uint16_t(ro); r[k] = uint16_t(rr); c[k] = uint16_t(cc);
        }
  }
};

const InvMap& invmap(const Module& m) {
  static InvMap b1(true, 1, 1), bminus(true, -1, 2), bplus(true, 1, 2), fpix(false, -1, 0);
  if (!m.barrel) return fpix;
  if (m.layer == 1) return b1;
  return m.side == -1 ? bminus : bplus;
}

// Gain table parameters (decoded as ped = p*pedPrec + minPed, gain = g*gainPrec + minGain).
constexpr float kMinPed = 0.f, kMaxPed = 60.f, kMinGain = 1.8f, kMaxGain = 4.2f;
constexpr uint32_t kDeadFlag = 255, kNoisyFlag = 254;

uint8_t gain_code(int module, int col, int block) {
  uint32_t h = uint32_t(module) * 2654435761u ^ uint32_t(col * 40503 + block * 977);
  h ^= h >> 13; h *= 0x5bd1e995u; h ^= h >> 15;
  return uint8_t(60 + (h % 120));
}
uint8_t ped_code(int module, int col, int block) {
  uint32_t h = uint32_t(module) * 2246822519u ^ uint32_t(col * 3266489917u + block * 668265263u);
  h ^= h >> 15; h *= 0x27d4eb2fu; h ^= h >> 13;
  return uint8_t(40 + (h % 120));
}
float decode_gain(uint8_t g) { return float(g) * ((kMaxGain - kMinGain) / 254.f) + kMinGain; }
float decode_ped(uint8_t p) { return float(p) * ((kMaxPed - kMinPed) / 254.f) + kMinPed; }

struct Buf {
  std::vector<uint8_t> b;
  template <class T> void put(const T& v) { const uint8_t* p = reinterpret_cast<const uint8_t*>(&v); b.insert(b.end(), p, p + sizeof(T)); }
  void put_bytes(const void* p, size_t n) { const uint8_t* q = static_cast<const uint8_t*>(p); b.insert(b.end(), q, q + n); }
};

uint8_t* to_malloc(const std::vector<uint8_t>& v, size_t* n) {
  *n = v.size();
  uint8_t* p = static_cast<uint8_t*>(std::malloc(v.size() ? v.size() : 1));
  if (!v.empty()) std::memcpy(p, v.data(), v.size());
  return p;
}

// ---- pixel <-> local position (inverse of the CPE's local_x/local_y units) ----
int pixel_from_ux(double u) {  // u in local_x units [0,162)
  if (u < 0 || u >= 162) return -1;
  if (u < 79) return int(u);
  if (u < 81) return 79;
  if (u < 83) return 80;
  return int(u) - 2;
}
int pixel_from_uy(double u) {  // u in local_y units [0,432)
  if (u < 0 || u >= 432) return -1;
  int roc = int(u / 54.0);
  double w = u - roc * 54.0;
  int inroc;
  if (w < 2) inroc = 0;
  else if (w >= 52) inroc = 51;
  else inroc = int(w) - 1;
  return roc * 52 + inroc;
}

struct PixelDep { uint32_t key; float q; };  // key = module<<17 | row<<9 | col

struct EventGen {
  const Geometry& g = geom();
  std::mt19937_64 rng;
  std::vector<PixelDep> deps;
  double bs[3];
  explicit EventGen(uint64_t seed, const double* beamspot) : rng(seed) { for (int i = 0; i < 3; ++i) bs[i] = beamspot[i]; }
  double uni() { return std::uniform_real_distribution<double>(0.0, 1.0)(rng); }
  double gaus() { return std::normal_distribution<double>(0.0, 1.0)(rng); }

  // Moyal approximation to the Landau distribution, MPV 21k electrons for a normal crossing.
  double landau_charge() {
    double q;
    do {
      double x = gaus();
      double l = -2.0 * std::log(std::fabs(x) + 1e-12);  // chi2 ~ Moyal-like tail
      q = 21000.0 + 1800.0 * (l - 0.0) * 0.5;
    } while (q < 8000.0 || q > 120000.0);
    return q;
  }

  void deposit(int mod, const double* xl, const double* dl, double thick, double charge) {
    // straight segment through the sensor: centre xl, local direction dl (dl[2] != 0)
    const Module& m = g.mods[mod];
    (void)m;
    double tx = dl[0] / dl[2], ty = dl[1] / dl[2];
    const int K = 24;
    double qs = charge / K;
    for (int k = 0; k < K; ++k) {
      double f = (k + 0.5) / K - 0.5;
      double x = xl[0] + tx * thick * f, y = xl[1] + ty * thick * f;
      x += 0.0020 * gaus(); y += 0.0020 * gaus();  // diffusion
      int row = pixel_from_ux(x / kPitchX + 81.0);
      int col = pixel_from_uy(y / kPitchY + 216.0);
      if (row < 0 || col < 0) continue;
      deps.push_back({uint32_t(mod) << 17 | uint32_t(row) << 9 | uint32_t(col), float(qs)});
    }
  }

  // Helix from vertex v with (pt, eta, phi, q): propagate, find module crossings, deposit charge.
  void track(const double* v, double pt, double eta, double phi0, int q, double ineff) {
    double R = 1.0 / (kInvRadiusPerGeV / pt);  // cm
    double cot = std::sinh(eta);
    double cphi = std::cos(phi0), sphi = std::sin(phi0);
    // circle centre (counter-clockwise for q<0 in this convention)
    double cx = v[0] - q * R * sphi, cy = v[1] + q * R * cphi;
    auto pos_at = [&](double s, double* x) {  // s = transverse path length
      double a = s / R;
      double ang0 = std::atan2(v[1] - cy, v[0] - cx);
      double ang = ang0 + q * a;
      x[0] = cx + R * std::cos(ang); x[1] = cy + R * std::sin(ang); x[2] = v[2] + cot * s;
    };
    auto dir_at = [&](double s, double* d) {
      double a = s / R;
      double ang0 = std::atan2(v[1] - cy, v[0] - cx);
      double ang = ang0 + q * a;
      d[0] = -q * std::sin(ang); d[1] = q * std::cos(ang); d[2] = cot;
    };
    double path_scale = 1.0;
    // barrel crossings: solve |pos(s)| = r by bisection on s
    for (int L = 0; L < 4; ++L) {
      double r = kBarrelR[L];
      if (2 * R < r) continue;
      double lo = 0, hi = std::min(M_PI * R, 4 * r + 10);
      double x[3];
      pos_at(hi, x);
      if (std::hypot(x[0], x[1]) < r) continue;
      for (int it = 0; it < 60; ++it) {
        double mid = 0.5 * (lo + hi);
        pos_at(mid, x);
        if (std::hypot(x[0], x[1]) < r) lo = mid; else hi = mid;
      }
      double s = 0.5 * (lo + hi);
      pos_at(s, x);
      if (std::fabs(x[2]) > 26.0) continue;
      double d[3];
      dir_at(s, d);
      // candidate modules: nearest ladders in phi, module along z
      int nl = kLaddersPerLayer[L];
      double ph = std::atan2(x[1], x[0]);
      for (int dk = -1; dk <= 1; ++dk) {
        double kf = ph / (2 * M_PI) * nl - 0.25 * L;
        int k = ((int(std::lround(kf)) + dk) % nl + nl) % nl;
        int mz = int(std::floor((x[2] + 26.0) / 6.5));
        for (int dz = -1; dz <= 1; ++dz) {
          int z = mz + dz;
          if (z < 0 || z > 7) continue;
          int id = kLayerStart[L] + k * 8 + z;
          hit_module(id, x, d, kThickB, ineff, &path_scale);
        }
      }
    }
    // endcap crossings
    if (std::fabs(cot) > 1e-6) {
      for (int s = 0; s < 2; ++s) {
        for (int dd = 0; dd < 3; ++dd) {
          double zd = (s == 0 ? 1.0 : -1.0) * kDiskZ[dd];
          double sp = (zd - v[2]) / cot;
          if (sp <= 0 || sp > M_PI * R) continue;
          double x[3], d[3];
          pos_at(sp, x);
          dir_at(sp, d);
          double r = std::hypot(x[0], x[1]);
          if (r < 3.5 || r > 16.5) continue;
          int base = kLayerStart[4 + 3 * s + dd];
          double ph = std::atan2(x[1], x[0]);
          for (int ring = 0; ring < 2; ++ring) {
            int n = ring == 0 ? 44 : 68;
            int off = ring == 0 ? 0 : 44;
            double kf = ph / (2 * M_PI) * n - 0.5 * ring;
            for (int dk = -1; dk <= 1; ++dk) {
              int k = ((int(std::lround(kf)) + dk) % n + n) % n;
              hit_module(base + off + k, x, d, kThickE, ineff, &path_scale);
            }
          }
        }
      }
    }
  }

  // intersect the local straight line (point x, direction d) with module `id`'s plane
  void hit_module(int id, const double* x, const double* d, double thick, double ineff, double*) {
    const Module& m = g.mods[id];
    double v[3] = {x[0] - m.p[0], x[1] - m.p[1], x[2] - m.p[2]};
    double xl[3], dl[3];
    for (int i = 0; i < 3; ++i) {
      xl[i] = m.R[3 * i] * v[0] + m.R[3 * i + 1] * v[1] + m.R[3 * i + 2] * v[2];
      dl[i] = m.R[3 * i] * d[0] + m.R[3 * i + 1] * d[1] + m.R[3 * i + 2] * d[2];
    }
    if (std::fabs(dl[2]) < 1e-3) return;
    double t = -xl[2] / dl[2];
    double dn = std::sqrt(dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2]);
    if (std::fabs(t) * dn > 1.5) return;  // too far from the crossing point
    double p[2] = {xl[0] + t * dl[0], xl[1] + t * dl[1]};
    if (std::fabs(p[0]) > 0.80 || std::fabs(p[1]) > 3.22) return;
    if (uni() < ineff) return;
    double cosn = std::fabs(dl[2]) / dn;
    double q = landau_charge() / std::max(cosn, 0.05);
    double xc[3] = {p[0], p[1], 0.0};
    deposit(id, xc, dl, thick, q);
  }

  void noise(double occupancy) {
    double mean = occupancy * double(kModules) * kRows * kCols;
    int n = std::poisson_distribution<int>(mean)(rng);
    for (int i = 0; i < n; ++i) {
      uint32_t mod = uint32_t(uni() * kModules) % kModules;
      uint32_t row = uint32_t(uni() * kRows) % kRows;
      uint32_t col = uint32_t(uni() * kCols) % kCols;
      deps.push_back({mod << 17 | row << 9 | col, float(1500.0 + 3500.0 * uni())});
    }
  }
};

// electrons -> 8-bit ADC through the inverse of calib_digis (gpu_calib_pixel.jl:46-63)
int electrons_to_adc(int mod, int row, int col, double q) {
  int block = row / 80;
  double gain = decode_gain(gain_code(mod, col, block));
  double ped = decode_ped(ped_code(mod, col, block));
  double cf = mod < 96 ? 50.0 : 47.0, off = mod < 96 ? -670.0 : -60.0;
  double vcal = (q - off) / cf;
  double adc = vcal / gain + ped;
  int a = int(std::lround(adc));
  return std::max(1, std::min(255, a));
}

struct FedWords { std::vector<uint32_t> w; };

void pack_event(const std::vector<PixelDep>& deps_in, uint32_t event_number, Buf& out) {
  const Geometry& g = geom();
  // merge deposits per pixel
  std::vector<PixelDep> d = deps_in;
  std::sort(d.begin(), d.end(), [](const PixelDep& a, const PixelDep& b) { return a.key < b.key; });
  std::vector<PixelDep> px;
  for (size_t i = 0; i < d.size();) {
    size_t j = i;
    double q = 0;
    while (j < d.size() && d[j].key == d[i].key) q += d[j++].q;
    if (q >= 1000.0) px.push_back({d[i].key, float(q)});
    i = j;
  }
  // per link / roc word lists
  int nfed = (kModules + kModulesPerFed - 1) / kModulesPerFed;
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> fed_words(nfed);  // (sort key, word)
  for (auto& p : px) {
    int mod = int(p.key >> 17), row = int((p.key >> 9) & 255), col = int(p.key & 511);
    const Module& m = g.mods[mod];
    const InvMap& im = invmap(m);
    int k = row * kCols + col;
    int roc_in_det = im.roc[k], rr = im.r[k], cc = im.c[k];
    int fed = mod / kModulesPerFed;
    int link = 2 * (mod % kModulesPerFed) + 1 + (roc_in_det >= 8 ? 1 : 0);
    int roc = (roc_in_det & 7) + 1;
    uint32_t adc = uint32_t(electrons_to_adc(mod, row, col, p.q));
    uint32_t w;
    if (m.barrel && m.layer == 1) {
      w = (uint32_t(link) << 26) | (uint32_t(roc) << 21) | (uint32_t(cc) << 15) | (uint32_t(rr) << 8) | adc;
    } else {
      uint32_t dcol = uint32_t(cc / 2), pxid = uint32_t(2 * (80 - rr) + (cc % 2));
      w = (uint32_t(link) << 26) | (uint32_t(roc) << 21) | (dcol << 16) | (pxid << 8) | adc;
    }
    uint32_t sk = (uint32_t(link) << 24) | (uint32_t(roc) << 20) | ((w >> 8) & 0xFFFF);
    fed_words[fed].push_back({sk, w});
  }
  int32_t nf = nfed;
  out.put(nf);
  for (int f = 0; f < nfed; ++f) {
    auto& fw = fed_words[f];
    std::sort(fw.begin(), fw.end());
    std::vector<uint32_t> words;
    words.reserve(fw.size() + 1);
    for (auto& e : fw) words.push_back(e.second);
    if (words.size() & 1) words.push_back(0u);  // FED payloads hold an even number of 32-bit words
    int32_t fed_id = kFedBase + f;
    uint32_t nwords64 = uint32_t(words.size() / 2 + 2);
    int32_t size = int32_t(nwords64 * 8);
    out.put(fed_id);
    out.put(size);
    uint32_t h0 = uint32_t(fed_id) << 8, h1 = (0x5u << 28) | (event_number & 0xFFFFFF);
    out.put(h0); out.put(h1);
    out.put_bytes(words.data(), words.size() * 4);
    uint32_t t0 = 0, t1 = (0xAu << 28) | (nwords64 & 0xFFFFFF);
    out.put(t0); out.put(t1);
  }
}

const double kBeamSpot[3] = {0.02, -0.01, 0.3};

}  // namespace

extern "C" {

int pxlgen_n_modules() { return kModules; }

// Conditions, each in the reference's binary layout. Buffers are malloc'ed;
// release them with pxlgen_free.
int pxlgen_conditions(uint8_t** cabling, size_t* n_cabling, uint8_t** fed_ids, size_t* n_fed_ids, uint8_t** gain,
                      size_t* n_gain, uint8_t** cpe, size_t* n_cpe, uint8_t** beamspot, size_t* n_beamspot) {
  const Geometry& g = geom();
  // cabling map: 6 x 57600 u32 + 57600 u8 + u32 n + n u8
  std::vector<uint32_t> fed(kCablingSize), link(kCablingSize), roc(kCablingSize), raw(kCablingSize, 9999u),
      rocdet(kCablingSize), modid(kCablingSize, 9999u);
  std::vector<uint8_t> bad(kCablingSize, 0);
  for (int m = 0; m < kModules; ++m) {
    int f = m / kModulesPerFed;
    for (int half = 0; half < 2; ++half) {
      int l = 2 * (m % kModulesPerFed) + 1 + half;
      for (int r = 1; r <= 8; ++r) {
        int idx = f * kMaxLink * kMaxRoc + (l - 1) * kMaxRoc + r;  // C index of element (fed, link, roc)
        if (idx >= kCablingSize) continue;
        fed[idx] = uint32_t(f); link[idx] = uint32_t(l); roc[idx] = uint32_t(r);
        raw[idx] = g.mods[m].raw_id; rocdet[idx] = uint32_t(half * 8 + r - 1); modid[idx] = uint32_t(m);
      }
    }
  }
  Buf cb;
  cb.put_bytes(fed.data(), 4 * kCablingSize); cb.put_bytes(link.data(), 4 * kCablingSize);
  cb.put_bytes(roc.data(), 4 * kCablingSize); cb.put_bytes(raw.data(), 4 * kCablingSize);
  cb.put_bytes(rocdet.data(), 4 * kCablingSize); cb.put_bytes(modid.data(), 4 * kCablingSize);
  cb.put_bytes(bad.data(), kCablingSize);
  uint32_t nunp = kModules;
  cb.put(nunp);
  std::vector<uint8_t> unp(kModules, 1);
  cb.put_bytes(unp.data(), unp.size());
  *cabling = to_malloc(cb.b, n_cabling);

  Buf fb;
  int nfed = (kModules + kModulesPerFed - 1) / kModulesPerFed;
  uint32_t nf = uint32_t(nfed);
  fb.put(nf);
  for (int f = 0; f < nfed; ++f) { uint32_t id = uint32_t(kFedBase + f); fb.put(id); }
  *fed_ids = to_malloc(fb.b, n_fed_ids);

  // gains: 8-byte skip, 2000 x {u32 first, u32 last, i32 cols}, 6 f32, 4 u32, u32 nbytes, {u8 gain, u8 ped}...
  Buf gb;
  uint64_t skip = 0;
  gb.put(skip);
  const uint32_t per_module = kCols * 2 * 2;  // bytes: 2 blocks of 80 rows per column, 2 bytes each
  for (int m = 0; m < 2000; ++m) {
    uint32_t first = m < kModules ? uint32_t(m) * per_module : 0, last = m < kModules ? first + per_module : 0;
    int32_t cols = m < kModules ? kCols : 1;
    gb.put(first); gb.put(last); gb.put(cols);
  }
  float fp[6] = {kMinPed, kMaxPed, kMinGain, kMaxGain, (kMaxPed - kMinPed) / 254.f, (kMaxGain - kMinGain) / 254.f};
  for (float v : fp) gb.put(v);
  uint32_t up[4] = {80u, 254u, kDeadFlag, kNoisyFlag};
  for (uint32_t v : up) gb.put(v);
  uint32_t nbytes = uint32_t(kModules) * per_module;
  gb.put(nbytes);
  for (int m = 0; m < kModules; ++m)
    for (int c = 0; c < kCols; ++c)
      for (int b = 0; b < 2; ++b) { uint8_t gg = gain_code(m, c, b), pp = ped_code(m, c, b); gb.put(gg); gb.put(pp); }
  *gain = to_malloc(gb.b, n_gain);

  // cpefast: 4 f32, u32 n, n x DetParams (112 bytes), 6x148 f32, 2 f32, 11 u32, 116 u8
  Buf pb;
  float cm[4] = {kThickB, kThickE, kPitchX, kPitchY};
  for (float v : cm) pb.put(v);
  uint32_t nd = kModules;
  pb.put(nd);
  for (int i = 0; i < kModules; ++i) {
    const Module& m = g.mods[i];
    uint8_t isb = m.barrel, ispz = m.p[2] > 0;
    uint16_t layer = uint16_t(m.barrel ? m.layer : 4 + m.layer), index = uint16_t(i);
    uint16_t pad = 0;
    pb.put(isb); pb.put(ispz); pb.put(layer); pb.put(index); pb.put(pad); pb.put(m.raw_id);
    float shiftX = m.barrel ? 0.0015f : 0.0002f, shiftY = 0.f;
    float cwX = m.barrel ? 0.0030f : 0.0004f, cwY = 0.f;
    pb.put(shiftX); pb.put(shiftY); pb.put(cwX); pb.put(cwY);
    pb.put(m.x0); pb.put(m.y0); pb.put(m.z0);
    float sx[3] = {0.0017f, 0.0028f, 0.0045f}, sy[3] = {0.0025f, 0.0042f, 0.0060f};
    for (float v : sx) pb.put(v);
    for (float v : sy) pb.put(v);
    for (int j = 0; j < 3; ++j) { float v = float(m.p[j]); pb.put(v); }
    for (int j = 0; j < 9; ++j) { float v = float(m.R[j]); pb.put(v); }
  }
  // average geometry over barrel ladders
  std::vector<float> lz(kLadders), lx(kLadders), ly(kLadders), lr(kLadders), lminz(kLadders), lmaxz(kLadders);
  for (int l = 0; l < kLadders; ++l) {
    double sx = 0, sy = 0, sz = 0, mn = 1e9, mx = -1e9;
    for (int k = 0; k < 8; ++k) {
      const Module& m = g.mods[l * 8 + k];
      sx += m.p[0]; sy += m.p[1]; sz += m.p[2];
      mn = std::min(mn, m.p[2] - 3.24); mx = std::max(mx, m.p[2] + 3.24);
    }
    lx[l] = float(sx / 8); ly[l] = float(sy / 8); lz[l] = float(sz / 8);
    lr[l] = float(std::hypot(sx / 8, sy / 8)); lminz[l] = float(mn); lmaxz[l] = float(mx);
  }
  pb.put_bytes(lz.data(), 4 * kLadders); pb.put_bytes(lx.data(), 4 * kLadders); pb.put_bytes(ly.data(), 4 * kLadders);
  pb.put_bytes(lr.data(), 4 * kLadders); pb.put_bytes(lminz.data(), 4 * kLadders); pb.put_bytes(lmaxz.data(), 4 * kLadders);
  float ecz[2] = {float(kDiskZ[0]), float(-kDiskZ[0])};
  pb.put(ecz[0]); pb.put(ecz[1]);
  for (int i = 0; i < 11; ++i) { uint32_t v = uint32_t(kLayerStart[i]); pb.put(v); }
  for (int i = 0; i < 116; ++i) {
    int det = i * 16, L = 0;
    while (L < 11 && det >= kLayerStart[L + 1]) ++L;
    uint8_t v = uint8_t(L);
    pb.put(v);
  }
  *cpe = to_malloc(pb.b, n_cpe);

  Buf bb;
  float bsv[11] = {float(kBeamSpot[0]), float(kBeamSpot[1]), float(kBeamSpot[2]), 5.0f, 0.0012f, 0.0012f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (float v : bsv) bb.put(v);
  *beamspot = to_malloc(bb.b, n_beamspot);
  return 0;
}

// Events.
//   mode 0: one vertex with `ntracks` tracks, no noise, no inefficiency
//   mode 1: `pu` vertices, Poisson(30) tracks each, 1e-4 noise, 1% inefficiency
//   mode 2: pileup uniform in [0, pu] per event (at least one vertex), as mode 1
// The blob holds the events back to back in raw.bin layout; offsets[n_events+1].
int pxlgen_events(uint64_t seed, int32_t n_events, int32_t mode, double pu, int32_t ntracks, int32_t n_threads,
                  uint8_t** blob, size_t* nbytes, uint64_t* offsets) {
  if (n_events < 0) return -1;
  std::vector<Buf> evbuf(n_events);
  int nt = n_threads > 0 ? n_threads : int(std::max(1u, std::thread::hardware_concurrency()));
  nt = std::max(1, std::min(nt, n_events > 0 ? n_events : 1));
  auto work = [&](int t) {
    for (int e = t; e < n_events; e += nt) {
      EventGen gen(seed * 1000003ull + uint64_t(e) * 7919ull + 17ull, kBeamSpot);
      int nvtx = mode == 0 ? 1 : (mode == 1 ? int(pu) : std::max(1, int(gen.uni() * (pu + 1))));
      for (int v = 0; v < nvtx; ++v) {
        double vz = kBeamSpot[2] + 5.0 * gen.gaus();
        double vtx[3] = {kBeamSpot[0] + 0.0012 * gen.gaus(), kBeamSpot[1] + 0.0012 * gen.gaus(), vz};
        int n = mode == 0 ? ntracks : std::poisson_distribution<int>(30.0)(gen.rng);
        for (int k = 0; k < n; ++k) {
          double invpt = 0.1 + 1.9 * gen.uni();
          double eta = -2.5 + 5.0 * gen.uni();
          double phi = -M_PI + 2 * M_PI * gen.uni();
          int q = gen.uni() < 0.5 ? -1 : 1;
          gen.track(vtx, 1.0 / invpt, eta, phi, q, mode == 0 ? 0.0 : 0.01);
        }
      }
      if (mode != 0) gen.noise(1e-4);
      pack_event(gen.deps, uint32_t(e + 1), evbuf[e]);
    }
  };
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) th.emplace_back(work, t);
  for (auto& t : th) t.join();
  size_t tot = 0;
  for (auto& b : evbuf) tot += b.b.size();
  uint8_t* p = static_cast<uint8_t*>(std::malloc(tot ? tot : 1));
  size_t o = 0;
  for (int e = 0; e < n_events; ++e) {
    offsets[e] = o;
    if (!evbuf[e].b.empty()) std::memcpy(p + o, evbuf[e].b.data(), evbuf[e].b.size());
    o += evbuf[e].b.size();
  }
  offsets[n_events] = o;
  *blob = p;
  *nbytes = tot;
  return 0;
}

void pxlgen_free(void* p) { std::free(p); }

// ---------------------------------------------------------------- fit workload
// Helices for the stand-alone fits: an 8-layer barrel telescope made of the four
// pixel layers above (hits there carry the module id, for alignment) and four
// outer cylinders at 20/24/28/32 cm, so that tracks of 6 to 8 hits exist.
// Hit count mix 30/40/20/10 % for 3/4/5/6-8 hits; 1/pT uniform in [0.1, 2] GeV^-1,
// |eta| < 1, z0 ~ N(0, 5 cm), transverse origin ~ N(0, 10 um); at every layer a
// multiple-scattering kink of 0.02 X0 (Highland), then the measured point is
// smeared by N(0, 10 um) along r-phi and N(0, 20 um) along z. Each track draws
// from its own counter-based random stream, so results do not depend on threads.
int32_t pxlgen_module_positions(double* out) {  // [1856][3] module centres (cm)
  const Geometry& g = geom();
  for (int m = 0; m < kModules; ++m)
    for (int j = 0; j < 3; ++j) out[3 * m + j] = g.mods[m].p[j];
  return kModules;
}

int32_t pxlgen_fit_tracks(uint64_t seed, int32_t n_tracks, int32_t n_threads, double* hits, float* ge,
                          int32_t* offsets, int16_t* module, double* truth) {
  if (n_tracks < 0 || !hits || !ge || !offsets || !module) return -1;
  static const double kR[8] = {2.9, 6.8, 10.9, 16.0, 20.0, 24.0, 28.0, 32.0};
  static const double kHalf[8] = {26.0, 26.0, 26.0, 26.0, 60.0, 60.0, 60.0, 60.0};
  const double s_rphi = 10e-4, s_z = 20e-4;
  struct Rng {  // splitmix64 stream
    uint64_t x;
    uint64_t next() { uint64_t z = (x += 0x9e3779b97f4a7c15ull); z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
                      z = (z ^ (z >> 27)) * 0x94d049bb133111ebull; return z ^ (z >> 31); }
    double uni() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    double gaus() { double u = uni(), v = uni(); return std::sqrt(-2.0 * std::log(u + 1e-300)) * std::cos(2 * M_PI * v); }
  };
  auto n_hits_of = [&](int64_t t) {
    Rng r{seed * 0x2545f4914f6cdd1dull + uint64_t(t) * 0x9e3779b97f4a7c15ull + 1};
    const double u = r.uni();
    if (u < 0.3) return 3;
    if (u < 0.7) return 4;
    if (u < 0.9) return 5;
    return 6 + int(r.uni() * 3.0);
  };
  offsets[0] = 0;
  for (int64_t t = 0; t < n_tracks; ++t) offsets[t + 1] = offsets[t] + n_hits_of(t);
  const Geometry& g = geom();
  (void)g;
  auto one = [&](int64_t t) {
    const int n = offsets[t + 1] - offsets[t];
    Rng r{seed * 0x94d049bb133111ebull + uint64_t(t) * 0xbf58476d1ce4e5b9ull + 7};
    double hx[8], hy[8], hz[8];
    double tr[5] = {0, 0, 0, 0, 0};
    for (int attempt = 0; attempt < 1000; ++attempt) {
      const double invpt = 0.1 + 1.9 * r.uni();
      const double eta = attempt < 900 ? -1.0 + 2.0 * r.uni() : 0.0;
      const double phi0 = -M_PI + 2 * M_PI * r.uni();
      const int q = r.uni() < 0.5 ? -1 : 1;
      const double z0 = 5.0 * r.gaus();
      double px = 0.001 * r.gaus(), py = 0.001 * r.gaus(), pz = z0;
      const double p = std::cosh(eta) / invpt;  // |p| in GeV
      double theta = 2.0 * std::atan(std::exp(-eta));
      double phid = phi0;                        // direction of motion in the transverse plane
      tr[0] = phi0; tr[1] = 0.0; tr[2] = q * invpt; tr[3] = std::sinh(eta); tr[4] = z0;
      bool ok = true;
      for (int L = 0; L < n && ok; ++L) {
        const double pt = p * std::sin(theta);
        const double R = pt / kInvRadiusPerGeV;  // cm
        const double cot = std::cos(theta) / std::sin(theta);
        const double cx = px + q * R * (-std::sin(phid)), cy = py + q * R * std::cos(phid);
        const double dc = std::hypot(cx, cy), rl = kR[L];
        if (dc + R < rl || std::fabs(dc - R) > rl || dc == 0) { ok = false; break; }
        const double a = (rl * rl - R * R + dc * dc) / (2 * dc);
        const double h = std::sqrt(std::max(rl * rl - a * a, 0.0));
        const double ux = cx / dc, uy = cy / dc;
        const double psi0 = std::atan2(py - cy, px - cx);
        double best = 1e300, bx = 0, by = 0;
        for (int sg = -1; sg <= 1; sg += 2) {
          const double ix = a * ux - sg * h * uy, iy = a * uy + sg * h * ux;
          double dpsi = q * (std::atan2(iy - cy, ix - cx) - psi0);
          while (dpsi <= 1e-12) dpsi += 2 * M_PI;
          while (dpsi > 2 * M_PI) dpsi -= 2 * M_PI;
          if (dpsi < best) { best = dpsi; bx = ix; by = iy; }
        }
        if (best > M_PI) { ok = false; break; }  // would have to loop back
        const double sT = R * best;
        px = bx; py = by; pz += cot * sT;
        if (std::fabs(pz) > kHalf[L]) { ok = false; break; }
        phid += q * best;
        hx[L] = px; hy[L] = py; hz[L] = pz;
        // Highland kink for 0.02 X0 crossed at the track's polar angle
        const double x0 = 0.02 / std::sin(theta);
        const double th0 = 0.0136 / p * std::sqrt(x0) * (1.0 + 0.038 * std::log(x0));
        phid += th0 * r.gaus() / std::sin(theta);
        theta += th0 * r.gaus();
        if (theta <= 0.05 || theta >= M_PI - 0.05) { ok = false; break; }
      }
      if (ok) break;
    }
    const int64_t b = offsets[t];
    for (int L = 0; L < n; ++L) {
      const double ph = std::atan2(hy[L], hx[L]);
      const double sn = std::sin(ph), cs = std::cos(ph);
      const double d1 = s_rphi * r.gaus(), d2 = s_z * r.gaus();
      double* H = hits + 3 * (b + L);
      H[0] = hx[L] - sn * d1; H[1] = hy[L] + cs * d1; H[2] = hz[L] + d2;
      float* G = ge + 6 * (b + L);
      G[0] = float(s_rphi * s_rphi * sn * sn); G[1] = float(-s_rphi * s_rphi * sn * cs);
      G[2] = float(s_rphi * s_rphi * cs * cs); G[3] = 0.f; G[4] = 0.f; G[5] = float(s_z * s_z);
      int16_t mid = -1;
      if (L < 4) {
        const int nl = kLaddersPerLayer[L];
        const double kf = ph / (2 * M_PI) * nl - 0.25 * L;
        const int k = ((int(std::lround(kf))) % nl + nl) % nl;
        int mz = int(std::floor((hz[L] + 26.0) / 6.5));
        mz = mz < 0 ? 0 : (mz > 7 ? 7 : mz);
        mid = int16_t(kLayerStart[L] + k * 8 + mz);
      }
      module[b + L] = mid;
    }
    if (truth)
      for (int k = 0; k < 5; ++k) truth[5 * t + k] = tr[k];
  };
  int nt = n_threads > 0 ? n_threads : int(std::max(1u, std::thread::hardware_concurrency()));
  nt = std::max(1, std::min<int>(nt, n_tracks > 0 ? n_tracks : 1));
  std::vector<std::thread> th;
  for (int w = 0; w < nt; ++w)
    th.emplace_back([&, w] { for (int64_t t = w; t < n_tracks; t += nt) one(t); });
  for (auto& x : th) x.join();
  return offsets[n_tracks];
}

}  // extern "C"
