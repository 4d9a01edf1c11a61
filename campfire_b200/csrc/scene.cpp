// Seeded synthetic scenes for the benchmark workloads (host code).
//
// Domain: width x (dx * ny) with dx = width / nx (0.8 m x 1.2 m at 2:3 grids).
// Wood: the reference has square pieces only (common.wgsl:47-53), so a log of
// radius r becomes the square of equal cross-section area (half-side
// r*sqrt(pi)/2) at the same centre: squares of half-side r would overlap where
// the circles only come close, sealing cavities against the floor in which the
// pressure equation has no solution. Pieces are frozen (alive, zero velocity),
// every face at 600 K injecting fuel at the scene's flux (piece packing of
// js/main.js:196-199).
// Initial gas: T = 300 + 1500 exp(-r^2 / (2 * 0.05^2)) around (0.40, 0.12) m,
// Y_F = 0.3 of the same Gaussian, Y_O = YOamb (1 - Y_F), Y_S = 0, Y_P the rest;
// U, V uniform in [-0.01, 0.01] m/s from a counter-based hash of the seed.
// dt = min(2 ms, 0.5 dx / max|u|).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/campfire_gas.h"
#include "engine.h"

namespace {

uint64_t splitmix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// uniform in [0, 1) from (seed, stream, index): order-independent
double hash01(uint64_t seed, uint64_t stream, uint64_t k) {
  return (double)(splitmix(splitmix(seed ^ (stream * 0xD1B54A32D192ED03ull)) + k) >> 11) * (1.0 / 9007199254740992.0);
}
struct Rng {
  uint64_t seed, stream, n = 0;
  double u() { return hash01(seed, stream, n++); }
  double u(double a, double b) { return a + (b - a) * u(); }
};

struct Box { double x, y, a, h; };

void corners(const Box& b, double cx[4], double cy[4]) {
  const double c = std::cos(b.a), s = std::sin(b.a);
  const double lx[4] = {-b.h, b.h, b.h, -b.h}, ly[4] = {-b.h, -b.h, b.h, b.h};
  for (int k = 0; k < 4; k++) { cx[k] = b.x + c * lx[k] - s * ly[k]; cy[k] = b.y + s * lx[k] + c * ly[k]; }
}
// separating-axis test between two rotated squares, with a clearance margin
bool overlap(const Box& p, const Box& q, double margin) {
  double px[4], py[4], qx[4], qy[4];
  corners(p, px, py); corners(q, qx, qy);
  const double axes[4][2] = {{std::cos(p.a), std::sin(p.a)}, {-std::sin(p.a), std::cos(p.a)},
                             {std::cos(q.a), std::sin(q.a)}, {-std::sin(q.a), std::cos(q.a)}};
  for (auto& ax : axes) {
    double pmin = 1e30, pmax = -1e30, qmin = 1e30, qmax = -1e30;
    for (int k = 0; k < 4; k++) {
      const double dp = px[k] * ax[0] + py[k] * ax[1], dq = qx[k] * ax[0] + qy[k] * ax[1];
      pmin = std::min(pmin, dp); pmax = std::max(pmax, dp); qmin = std::min(qmin, dq); qmax = std::max(qmax, dq);
    }
    if (pmax + margin < qmin || qmax + margin < pmin) return false;
  }
  return true;
}
bool inside(const Box& b, double W, double H) {
  double cx[4], cy[4];
  corners(b, cx, cy);
  for (int k = 0; k < 4; k++) if (cx[k] < 0.005 || cx[k] > W - 0.005 || cy[k] < -1e-9 || cy[k] > H - 0.005) return false;
  return true;
}
bool fits(const Box& b, const std::vector<Box>& placed, double W, double H) {
  if (!inside(b, W, H)) return false;
  // keep 6 mm of gas between pieces: narrower seams close under the fractional
  // faces of a 1.5 mm grid and would seal cavities
  for (auto& q : placed) if (overlap(b, q, 0.006)) return false;
  return true;
}

}  // namespace

extern "C" int cfg_scene_generate(int kind, int nx, int ny, double width, uint64_t seed, float* T, float* Y, float* U,
                                  float* V, float* pieces, int* npieces, cfg_params* params, double* dt) {
  if (kind < 0 || kind > 2) return cfg::fail(CFG_ERR_INVAL, "scene kind must be 0, 1 or 2");
  if (nx < 2 || ny < 2 || !(width > 0)) return cfg::fail(CFG_ERR_INVAL, "bad grid");
  const double dx = width / nx, H = dx * ny;
  Rng rng{seed, 7};
  // ---- parameters
  cfg_params P;
  cfg::default_params(&P);
  const double Tamb = 300.0;
  double YOamb = 0.233, Bmul = 1.0, flux = 5e-3;
  if (kind == 1) flux = 8e-3;
  if (kind == 2) {
    Bmul = std::exp(rng.u(std::log(0.5), std::log(2.0)));
    YOamb = rng.u(0.18, 0.233);
  }
  P.Tamb = (float)Tamb;
  P.rhoAmb = (float)(101325.0 * 0.0289 / (8.314462 * Tamb));
  P.YOamb = (float)YOamb;
  P.reactB = (float)(2.0e10 * Bmul);
  P.reactTa = 15000.f; P.dHc = 15.0e6f; P.Pr = 0.7f; P.exchAlpha = 0.05f; P.depth = 0.3f;
  // ---- wood
  std::vector<Box> boxes;
  const double area_half = 0.5 * std::sqrt(3.14159265358979323846);   // half-side / radius at equal area
  if (kind == 0) {
    const double hf = 0.025 * area_half;
    boxes = {{0.35, 0.025, 0.0, hf}, {0.45, 0.025, 0.0, hf}, {0.40, 0.068, 0.0, hf}};
  } else if (kind == 1) {
    const double hf = 0.05 * area_half, cx = 0.5 * width;
    for (int k = 0; k < 5; k++) {
      for (int attempt = 0; attempt < 4000; attempt++) {
        Box b{};
        const double sg = (k % 2 == 0) ? -1.0 : 1.0;
        if (k < 2) b = Box{cx + sg * rng.u(0.13, 0.17), hf, 0.0, hf};
        else if (k < 4) b = Box{cx + sg * rng.u(0.04, 0.08), rng.u(0.12, 0.17), -sg * rng.u(0.45, 0.75), hf};
        else b = Box{cx + rng.u(-0.02, 0.02), rng.u(0.24, 0.30), rng.u(-0.3, 0.3), hf};
        if (fits(b, boxes, width, H)) { boxes.push_back(b); break; }
      }
    }
  } else {
    const int want = 2 + std::min(4, (int)(rng.u() * 5));
    for (int k = 0; k < want; k++) {
      const double hf = (rng.u() < 0.5 ? 0.025 : 0.05) * area_half;
      for (int attempt = 0; attempt < 2000; attempt++) {
        Box b{rng.u(0.05 + hf, width - 0.05 - hf), hf, 0.0, hf};
        bool ok = fits(b, boxes, width, H);
        for (auto& q : boxes) ok = ok && std::fabs(b.x - q.x) >= b.h + q.h + 0.01;
        if (ok) { boxes.push_back(b); break; }
      }
    }
  }
  const int np = (int)boxes.size();
  if (pieces) {
    std::memset(pieces, 0, sizeof(float) * CFG_MAX_PIECES * CFG_PIECE_FLOATS);
    for (int n = 0; n < np; n++) {
      float* p = pieces + n * CFG_PIECE_FLOATS;
      p[0] = (float)boxes[n].x; p[1] = (float)boxes[n].y; p[2] = (float)boxes[n].a; p[3] = (float)boxes[n].h;
      p[7] = 1.f;
      for (int f = 0; f < 4; f++) { p[8 + f] = 600.f; p[12 + f] = (float)flux; p[16 + f] = 0.f; }
    }
  }
  if (npieces) *npieces = np;
  P.nPieces = np;
  // ---- initial gas state
  const double s2 = 2.0 * 0.05 * 0.05;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      const double x = (i + 0.5) * dx - 0.40, y = (j + 0.5) * dx - 0.12;
      const double g = std::exp(-(x * x + y * y) / s2);
      const double yf = 0.3 * g, yo = YOamb * (1.0 - yf), ys = 0.0, yp = 1.0 - yf - yo - ys;
      const size_t k = (size_t)j * nx + i;
      if (T) T[k] = (float)(300.0 + 1500.0 * g);
      if (Y) { Y[4 * k] = (float)yf; Y[4 * k + 1] = (float)yo; Y[4 * k + 2] = (float)yp; Y[4 * k + 3] = (float)ys; }
    }
  double umax = 0.0;
  for (size_t k = 0; k < (size_t)(nx + 1) * ny; k++) {
    const double u = (2.0 * hash01(seed, 1, k) - 1.0) * 0.01;
    if (U) U[k] = (float)u;
    umax = std::max(umax, std::fabs((double)(float)u));
  }
  for (size_t k = 0; k < (size_t)nx * (ny + 1); k++) {
    const double v = (2.0 * hash01(seed, 2, k) - 1.0) * 0.01;
    if (V) V[k] = (float)v;
    umax = std::max(umax, std::fabs((double)(float)v));
  }
  const double dtv = umax > 0 ? std::min(2e-3, 0.5 * dx / umax) : 2e-3;
  if (dt) *dt = dtv;
  P.nx = nx; P.ny = ny; P.dx = (float)dx; P.dt = (float)dtv;
  if (params) *params = P;
  return CFG_OK;
}
