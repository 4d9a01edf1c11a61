// ORACLE — test infrastructure, not product code.
//
// CPU restatement of campfire's WGSL gas step (BoccheseGiacomo/campfire), used
// only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
// checker and as the timed CPU baseline. Nothing in the product links it.
//
// Parity status: the reference kernels are WGSL run by WebGPU in a browser; no
// JS engine and no WebGPU implementation exist on this machine, and the
// reference ships no golden vectors for these kernels. This restatement is
// pinned by (1) the hand-derived known answers in tests/test_oracle_known.py,
// (2) the 1D flame-speed known answer (flame1d.c, README.md:89), and (3) the
// fixtures in tests/golden/ produced by a mechanical WGSL->C++ translation of
// the reference's own shader text (oracle/wgsl2cpp.py).
//
// It follows, function by function (file:line cites in each comment):
//   shaders/common.wgsl     Params, Piece, idxC/idxU/idxV, rhoOf, muOf, rhoDOf, ambY, sdBox, faceOf
//   js/gpu.js:16-65         bilinear samplers f_/s_/mm_ with the boundary rules
//   shaders/advect.wgsl     trace, velForward, velCorrect, scalForward, scalCorrect
//   shaders/diffuse.wgsl    main
//   shaders/sources.wgsl    main (+ 8x8 workgroup tree reduction of the globals)
//   shaders/forces.wgsl     main
//   shaders/pressure.wgsl   coef, rhs0, coefRestrict, stencil, relax, residual,
//                           restrictRes, prolong, coarsest, project
//   shaders/geometry.wgsl   nearest, main
//   shaders/radiation.wgsl  planck580, hitBox, gasAt, main
//   js/fluid.js             levels :70-91, reset :162-176, writeParams/diffSub
//                           :180-199, encodeStep :225-253, vcycle :294-312,
//                           encodeReadback :315-324
//
// Templated on the arithmetic type R: R=float reproduces the WGSL f32
// arithmetic operation by operation (compile with -ffp-contract=off); R=double
// is the FP64 accuracy oracle for the same problem (the f32 parameter values
// promoted to double).
//
// Additions that the reference does not have, applied identically on the GPU:
//   * pressure solve modes: a fixed number of V(2,2) cycles (the reference runs
//     one, js/fluid.js:250), cycles until ||r||2/||rhs||2 <= tol, and an FP64
//     defect-correction loop around FP32 V-cycles;
//   * optional CFL time step dt = min(dt_cap, cfl*dx/max|u|) re-evaluated after
//     each step; with cfl = 0 the step is fixed, as in the reference;
//   * the multigrid level cap is 7 instead of 6 (js/fluid.js:72) so that
//     512x768 has a coarsest level of <= 256 cells;
//   * the ray count of the radiation pass is a parameter (64 in the reference,
//     radiation.wgsl:22).
#pragma once
#include <algorithm>
#include <cfenv>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace cforc {

// js/fluid.js:5-11
constexpr int MAX_PIECES = 64, PIECE_FLOATS = 20, ACC_GLOBAL = 512, ACC_LEN = ACC_GLOBAL + 16;
constexpr int N_FLOOR = 64, RAD_LEN = MAX_PIECES * 4 + N_FLOOR;
constexpr uint32_t SOLID_NONE = 0xffffffffu;   // common.wgsl:27
constexpr int MAX_LEVELS = 7;

// common.wgsl:4-15 (the 40-field uniform; field order is the upload order of js/fluid.js:13-24)
struct ParamsPOD {
  int32_t nx, ny; float dx, dt;
  float Tamb, rhoAmb, YOamb, grav;
  float cp, Pr, viscMult, diffMult;
  float reactB, reactTa, dHc, sO2;
  float sootFormA, sootFormTa, sootOxA, sootOxTa;
  float kappaSootC, kappaGas, exchAlpha, depth;
  float charA, charTa; int32_t nPieces; uint32_t frame;
  float heaterX0, heaterX1, heaterY1, heaterT;
  float burnerX0, burnerX1, burnerFlux, burnerT;
  float sootDensity, sigma, charO2, time;
};
static_assert(sizeof(ParamsPOD) == 160, "Params is 40 x 4 bytes");

// js/config.js:12-47 (PHYS) and the FluidSim defaults of js/fluid.js:35-45
struct Phys {
  static constexpr double Tamb = 293.15, p0 = 101325, Wmix = 0.0289, R = 8.314462, g = 9.81;
  static constexpr double YO2air = 0.232, cp = 1300, Pr = 0.7, dHc = 15.0e6, dHO2 = 13.1e6;
  static constexpr double reactB = 2.0e10, reactTa = 15000, sootFormA = 6.0e6, sootFormTa = 25000;
  static constexpr double sootOxA = 5.4e8, sootOxTa = 19800, sootDensity = 1800, kappaSootC = 1862;
  static constexpr double kappaGas = 0.8, exchAlpha = 0.05, charA = 6.6, charTa = 5800, charO2 = 2.667;
  static constexpr double sigma = 5.670374e-8;
  static double rhoAmb() { return p0 * Wmix / (R * Tamb); }
  static double sO2() { return dHc / dHO2; }
};

inline void default_params(ParamsPOD& p) {
  std::memset(&p, 0, sizeof p);
  p.Tamb = (float)Phys::Tamb; p.rhoAmb = (float)Phys::rhoAmb(); p.YOamb = (float)Phys::YO2air; p.grav = (float)Phys::g;
  p.cp = (float)Phys::cp; p.Pr = (float)Phys::Pr; p.viscMult = 1; p.diffMult = 1;
  p.reactB = (float)Phys::reactB; p.reactTa = (float)Phys::reactTa; p.dHc = (float)Phys::dHc; p.sO2 = (float)Phys::sO2();
  p.sootFormA = (float)Phys::sootFormA; p.sootFormTa = (float)Phys::sootFormTa;
  p.sootOxA = (float)Phys::sootOxA; p.sootOxTa = (float)Phys::sootOxTa;
  p.kappaSootC = (float)Phys::kappaSootC; p.kappaGas = (float)Phys::kappaGas; p.exchAlpha = (float)Phys::exchAlpha;
  p.depth = 0.8f; p.charA = (float)Phys::charA; p.charTa = (float)Phys::charTa;
  p.burnerT = 600; p.sootDensity = (float)Phys::sootDensity; p.sigma = (float)Phys::sigma; p.charO2 = (float)Phys::charO2;
}

// WGSL round(): nearest, ties to even; i32(f): truncation toward zero, saturating.
inline int32_t wgsl_i32(double v) {
  if (!(v == v)) return 0;
  if (v >= 2147483647.0) return INT32_MAX;
  if (v <= -2147483648.0) return INT32_MIN;
  return (int32_t)v;
}
template <class R> inline int32_t wgsl_i32_round(R v) { return wgsl_i32((double)std::nearbyint(v)); }

template <class R> struct Vec2 { R x, y; };
template <class R> struct Vec4 { R x, y, z, w; };
template <class R> inline Vec4<R> v4(R a, R b, R c, R d) { return Vec4<R>{a, b, c, d}; }
template <class R> inline Vec4<R> operator+(Vec4<R> a, Vec4<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
template <class R> inline Vec4<R> operator-(Vec4<R> a, Vec4<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
template <class R> inline Vec4<R> operator*(R s, Vec4<R> a) { return {s * a.x, s * a.y, s * a.z, s * a.w}; }
template <class R> inline Vec4<R> operator*(Vec4<R> a, R s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
template <class R> inline Vec4<R> operator*(Vec4<R> a, Vec4<R> b) { return {a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
template <class R> inline Vec4<R> operator/(Vec4<R> a, R s) { return {a.x / s, a.y / s, a.z / s, a.w / s}; }
template <class R> inline Vec4<R> vmax(Vec4<R> a, Vec4<R> b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z), std::max(a.w, b.w)}; }
template <class R> inline Vec4<R> vmin(Vec4<R> a, Vec4<R> b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z), std::min(a.w, b.w)}; }
// WGSL mix(a, b, t) = a * (1 - t) + b * t
template <class R> inline R mix(R a, R b, R t) { return a * (R(1) - t) + b * t; }
template <class R> inline Vec4<R> mix(Vec4<R> a, Vec4<R> b, R t) { return {mix(a.x, b.x, t), mix(a.y, b.y, t), mix(a.z, b.z, t), mix(a.w, b.w, t)}; }
template <class R> inline R clampv(R e, R lo, R hi) { return std::min(std::max(e, lo), hi); }
template <class R> inline R fract(R x) { return x - std::floor(x); }

// One piece as laid out in the storage buffer (common.wgsl:17-23)
struct PieceF { float pos[2], angle, half, vel[2], omega, alive, Ts[4], mflux[4], charCov[4]; };
static_assert(sizeof(PieceF) == PIECE_FLOATS * 4, "Piece is 20 floats");

enum SolverMode { SOLVE_FIXED = 0, SOLVE_TOL = 1, SOLVE_FP64 = 2 };

template <class R>
struct Sim {
  int nx = 0, ny = 0;
  double dxd = 0, dtd = 0, width = 0;   // the JS doubles (js/fluid.js:29-32)
  double dt_cap = 0, cfl = 0;           // CFL step (extension); cfl = 0 keeps dt fixed
  double time = 0; uint32_t frame = 0;
  std::string err;
  ParamsPOD P{};       // the uploaded uniform
  ParamsPOD host{};    // FluidSim.params (applied by write_params)
  float pieces[MAX_PIECES * PIECE_FLOATS] = {};
  int nray = 64;

  std::vector<R> U, Uh, U2, V, Vh, V2, T, Th, T2, fx, fy;
  std::vector<Vec4<R>> Y, Yh, Y2;
  std::vector<Vec2<R>> SQ;
  std::vector<R> gsdf; std::vector<uint32_t> gid;   // cellG = (sdf, bitcast id)
  int32_t faceW[MAX_PIECES * 4] = {};
  int32_t acc[ACC_LEN] = {};
  float rad[RAD_LEN * 4] = {};

  struct Level { int nx, ny; double h; R h2; std::vector<R> p, rhs, ax, ay; };
  std::vector<Level> lv;
  int diffSub = 1; R diffDt = 0;

  // pressure solve control (extension)
  int mode = SOLVE_FIXED, ncycles = 1, max_cycles = 50, min_cycles = 1;
  double tol = 1e-6;
  int last_cycles = 0; double last_rel = 0, last_rel0 = 0;
  // direct coarse solve of the TOL/FP64 modes (extension of the library; the reference
  // runs one fixed cycle with the 120-sweep coarsest level)
  int coarse_direct = 0;
  int krylov = 0;   // FP64 mode: flexible preconditioned CG around the FP32 V-cycle (extension)
  long w_cells = 0; // cycle shape of the solve loop (extension): the W tail (cycle_at)
  std::vector<R> cinv;
  bool cinv_ok = false;
  std::vector<double> p64, rhs64;   // FP64 defect correction state (level 0)

  // converted parameters (R)
  R dx, dt, Tamb, rhoAmb, YOamb, grav, cp, Pr, viscMult, diffMult, reactB, reactTa, dHc, sO2;
  R sootFormA, sootFormTa, sootOxA, sootOxTa, kappaSootC, kappaGas, exchAlpha, depth, charA, charTa;
  R heaterX0, heaterX1, heaterY1, heaterT, burnerX0, burnerX1, burnerFlux, burnerT, sootDensity, sigma, charO2;

  // ---------------------------------------------------------------- setup
  // FluidSim constructor + init (js/fluid.js:27-160)
  void create(int nx_, int ny_, double width_, double dt_) {
    nx = nx_; ny = ny_; width = width_;
    dxd = width / nx; dtd = dt_; dt_cap = dt_;
    default_params(host);
    const size_t nC = (size_t)nx * ny, nU = (size_t)(nx + 1) * ny, nV = (size_t)nx * (ny + 1);
    for (auto* a : {&U, &Uh, &U2}) a->assign(nU, R(0));
    for (auto* a : {&V, &Vh, &V2}) a->assign(nV, R(0));
    for (auto* a : {&T, &Th, &T2}) a->assign(nC, R(0));
    for (auto* a : {&Y, &Yh, &Y2}) a->assign(nC, Vec4<R>{0, 0, 0, 0});
    SQ.assign(nC, Vec2<R>{0, 0});
    gsdf.assign(nC, R(0)); gid.assign(nC, 0u);
    fx.assign(nU, R(0)); fy.assign(nV, R(0));
    // multigrid hierarchy (js/fluid.js:70-91), cap raised from 6 to 7 levels
    lv.clear();
    int lx = nx, ly = ny; double h = dxd;
    for (int l = 0; l < MAX_LEVELS; l++) {
      Level L; L.nx = lx; L.ny = ly; L.h = h; L.h2 = R((float)(h * h));
      L.p.assign((size_t)lx * ly, R(0)); L.rhs.assign((size_t)lx * ly, R(0));
      L.ax.assign((size_t)(lx + 1) * ly, R(0)); L.ay.assign((size_t)lx * (ly + 1), R(0));
      lv.push_back(std::move(L));
      if (lx % 2 || ly % 2 || lx * ly <= 256) break;
      lx /= 2; ly /= 2; h *= 2;
    }
    if (lv.back().nx * lv.back().ny > 256) throw std::runtime_error("coarsest level too large");
    p64.assign(nC, 0.0); rhs64.assign(nC, 0.0);
    write_params();
    reset();
  }

  // js/fluid.js:162-176
  void reset() {
    cinv_ok = false;
    std::fill(T.begin(), T.end(), R((float)Phys::Tamb));
    T2 = T; Th = T;
    const Vec4<R> y0{R(0), R(host.YOamb), R(0), R(0)};
    for (auto* a : {&Y, &Y2, &Yh}) std::fill(a->begin(), a->end(), y0);
    for (auto* a : {&U, &Uh, &U2, &V, &Vh, &V2}) std::fill(a->begin(), a->end(), R(0));
    std::fill(SQ.begin(), SQ.end(), Vec2<R>{0, 0});
    std::memset(acc, 0, sizeof acc); std::memset(rad, 0, sizeof rad);
    for (auto& L : lv) std::fill(L.p.begin(), L.p.end(), R(0));
    std::fill(p64.begin(), p64.end(), 0.0);
    time = 0;
  }

  // js/fluid.js:180-199 (+ conversion of the f32 uniform to R)
  void write_params() {
    host.nx = nx; host.ny = ny; host.dx = (float)dxd; host.dt = (float)dtd;
    host.time = (float)time; host.frame = frame;
    P = host;
    // explicit diffusion stability: dt_sub <= dx^2 / (4.5 alpha_max)  (js/fluid.js:190-198, JS doubles)
    const double Tmax = 2200, mu = 1.716e-5 * std::pow(Tmax / 273.15, 1.5) * 383.55 / (Tmax + 110.4);
    const double alpha = mu / Phys::Pr * (double)host.diffMult / (Phys::rhoAmb() * Phys::Tamb / Tmax);
    int n = (int)std::ceil(dtd / (dxd * dxd / (4.5 * alpha)));
    n = std::min(5, n % 2 ? n : n + 1);
    diffSub = n;
    diffDt = R((float)(dtd / n));
    convert();
  }

  void convert() {
    dx = R(P.dx); dt = R(P.dt); Tamb = R(P.Tamb); rhoAmb = R(P.rhoAmb); YOamb = R(P.YOamb); grav = R(P.grav);
    cp = R(P.cp); Pr = R(P.Pr); viscMult = R(P.viscMult); diffMult = R(P.diffMult); reactB = R(P.reactB);
    reactTa = R(P.reactTa); dHc = R(P.dHc); sO2 = R(P.sO2); sootFormA = R(P.sootFormA); sootFormTa = R(P.sootFormTa);
    sootOxA = R(P.sootOxA); sootOxTa = R(P.sootOxTa); kappaSootC = R(P.kappaSootC); kappaGas = R(P.kappaGas);
    exchAlpha = R(P.exchAlpha); depth = R(P.depth); charA = R(P.charA); charTa = R(P.charTa);
    heaterX0 = R(P.heaterX0); heaterX1 = R(P.heaterX1); heaterY1 = R(P.heaterY1); heaterT = R(P.heaterT);
    burnerX0 = R(P.burnerX0); burnerX1 = R(P.burnerX1); burnerFlux = R(P.burnerFlux); burnerT = R(P.burnerT);
    sootDensity = R(P.sootDensity); sigma = R(P.sigma); charO2 = R(P.charO2);
  }

  // js/fluid.js:201-204
  void upload_pieces(const float* data, int n) {
    host.nPieces = n;
    std::memcpy(pieces, data, sizeof pieces);
  }
  const PieceF& piece(uint32_t n) const { return reinterpret_cast<const PieceF*>(pieces)[n]; }

  // ---------------------------------------------------------------- common.wgsl
  int idxC(int i, int j) const { return j * nx + i; }
  int idxU(int i, int j) const { return j * (nx + 1) + i; }
  int idxV(int i, int j) const { return j * nx + i; }
  R rhoOf(R t) const { return rhoAmb * Tamb / t; }                                     // :33
  R muOf(R t) const {                                                                  // :36-38
    return R(1.716e-5) * std::pow(t / R(273.15), R(1.5)) * R(273.15 + 110.4) / (t + R(110.4)) * viscMult;
  }
  R rhoDOf(R t) const {                                                                // :40-42
    return R(1.716e-5) * std::pow(t / R(273.15), R(1.5)) * R(273.15 + 110.4) / (t + R(110.4)) / Pr * diffMult;
  }
  Vec4<R> ambY() const { return Vec4<R>{R(0), YOamb, R(0), R(0)}; }                          // :44
  // :47-53
  R sdBox(R px, R py, const PieceF& pc) const {
    const R c = std::cos(R(pc.angle)), s = std::sin(R(pc.angle));
    const R dxp = px - R(pc.pos[0]), dyp = py - R(pc.pos[1]);
    const R lx = c * dxp + s * dyp, ly = -s * dxp + c * dyp;
    const R qx = std::abs(lx) - R(pc.half), qy = std::abs(ly) - R(pc.half);
    const R mx = std::max(qx, R(0)), my = std::max(qy, R(0));
    return std::sqrt(mx * mx + my * my) + std::min(std::max(qx, qy), R(0));
  }
  // :56-62
  uint32_t faceOf(R px, R py, const PieceF& pc) const {
    const R c = std::cos(R(pc.angle)), s = std::sin(R(pc.angle));
    const R dxp = px - R(pc.pos[0]), dyp = py - R(pc.pos[1]);
    const R lx = c * dxp + s * dyp, ly = -s * dxp + c * dyp;
    if (std::abs(lx) > std::abs(ly)) return lx > R(0) ? 0u : 2u;
    return ly > R(0) ? 1u : 3u;
  }

  // ---------------------------------------------------------------- samplers (js/gpu.js:16-65)
  // C fields: open sides/top sample the ambient, the floor is zero-gradient (:32-35)
  template <class F> R fC(const std::vector<F>& a, R amb, int i, int j) const {
    if (i < 0 || i >= nx || j >= ny) return amb;
    return a[idxC(i, std::max(j, 0))];
  }
  Vec4<R> fC4(const std::vector<Vec4<R>>& a, int i, int j) const {
    if (i < 0 || i >= nx || j >= ny) return ambY();
    return a[idxC(i, std::max(j, 0))];
  }
  R sC(const std::vector<R>& a, R amb, R gx, R gy) const {
    const R fxp = gx - R(0.5), fyp = gy - R(0.5);
    const R bx = std::floor(fxp), by = std::floor(fyp), tx = fxp - bx, ty = fyp - by;
    const int i = wgsl_i32((double)bx), j = wgsl_i32((double)by);
    return mix(mix(fC(a, amb, i, j), fC(a, amb, i + 1, j), tx), mix(fC(a, amb, i, j + 1), fC(a, amb, i + 1, j + 1), tx), ty);
  }
  Vec4<R> sC4(const std::vector<Vec4<R>>& a, R gx, R gy) const {
    const R fxp = gx - R(0.5), fyp = gy - R(0.5);
    const R bx = std::floor(fxp), by = std::floor(fyp), tx = fxp - bx, ty = fyp - by;
    const int i = wgsl_i32((double)bx), j = wgsl_i32((double)by);
    return mix(mix(fC4(a, i, j), fC4(a, i + 1, j), tx), mix(fC4(a, i, j + 1), fC4(a, i + 1, j + 1), tx), ty);
  }
  void mmC(const std::vector<R>& a, R amb, R gx, R gy, R& lo, R& hi) const {
    const int i = wgsl_i32((double)std::floor(gx - R(0.5))), j = wgsl_i32((double)std::floor(gy - R(0.5)));
    const R A = fC(a, amb, i, j), C = fC(a, amb, i + 1, j), D = fC(a, amb, i, j + 1), E = fC(a, amb, i + 1, j + 1);
    lo = std::min(std::min(A, C), std::min(D, E)); hi = std::max(std::max(A, C), std::max(D, E));
  }
  void mmC4(const std::vector<Vec4<R>>& a, R gx, R gy, Vec4<R>& lo, Vec4<R>& hi) const {
    const int i = wgsl_i32((double)std::floor(gx - R(0.5))), j = wgsl_i32((double)std::floor(gy - R(0.5)));
    const Vec4<R> A = fC4(a, i, j), C = fC4(a, i + 1, j), D = fC4(a, i, j + 1), E = fC4(a, i + 1, j + 1);
    lo = vmin(vmin(A, C), vmin(D, E)); hi = vmax(vmax(A, C), vmax(D, E));
  }
  // U: still ambient air outside, no-slip floor ghost (:44-46)
  R fU(const std::vector<R>& a, int i, int j) const {
    if (i < 0 || i > nx || j >= ny) return R(0);
    if (j < 0) return -a[idxU(i, 0)];
    return a[idxU(i, j)];
  }
  // V: still ambient air outside, clamp at the floor (:47-48)
  R fV(const std::vector<R>& a, int i, int j) const {
    if (i < 0 || i >= nx || j > ny) return R(0);
    return a[idxV(i, std::max(j, 0))];
  }
  R sU(const std::vector<R>& a, R gx, R gy) const {
    const R fxp = gx - R(0), fyp = gy - R(0.5);
    const R bx = std::floor(fxp), by = std::floor(fyp), tx = fxp - bx, ty = fyp - by;
    const int i = wgsl_i32((double)bx), j = wgsl_i32((double)by);
    return mix(mix(fU(a, i, j), fU(a, i + 1, j), tx), mix(fU(a, i, j + 1), fU(a, i + 1, j + 1), tx), ty);
  }
  R sV(const std::vector<R>& a, R gx, R gy) const {
    const R fxp = gx - R(0.5), fyp = gy - R(0);
    const R bx = std::floor(fxp), by = std::floor(fyp), tx = fxp - bx, ty = fyp - by;
    const int i = wgsl_i32((double)bx), j = wgsl_i32((double)by);
    return mix(mix(fV(a, i, j), fV(a, i + 1, j), tx), mix(fV(a, i, j + 1), fV(a, i + 1, j + 1), tx), ty);
  }
  void mmU(const std::vector<R>& a, R gx, R gy, R& lo, R& hi) const {
    const int i = wgsl_i32((double)std::floor(gx - R(0))), j = wgsl_i32((double)std::floor(gy - R(0.5)));
    const R A = fU(a, i, j), C = fU(a, i + 1, j), D = fU(a, i, j + 1), E = fU(a, i + 1, j + 1);
    lo = std::min(std::min(A, C), std::min(D, E)); hi = std::max(std::max(A, C), std::max(D, E));
  }
  void mmV(const std::vector<R>& a, R gx, R gy, R& lo, R& hi) const {
    const int i = wgsl_i32((double)std::floor(gx - R(0.5))), j = wgsl_i32((double)std::floor(gy - R(0)));
    const R A = fV(a, i, j), C = fV(a, i + 1, j), D = fV(a, i, j + 1), E = fV(a, i + 1, j + 1);
    lo = std::min(std::min(A, C), std::min(D, E)); hi = std::max(std::max(A, C), std::max(D, E));
  }

  // ---------------------------------------------------------------- advect.wgsl
  // :28 vel = (s_U, s_V) / dx ; :31-34 RK2 midpoint back-trace
  void vel(R gx, R gy, R& vx, R& vy) const { vx = sU(U, gx, gy) / dx; vy = sV(V, gx, gy) / dx; }
  void trace(R gx, R gy, R tdt, R& ox, R& oy) const {
    R vx, vy; vel(gx, gy, vx, vy);
    const R hd = R(0.5) * tdt;
    const R mx = gx - hd * vx, my = gy - hd * vy;
    vel(mx, my, vx, vy);
    ox = gx - tdt * vx; oy = gy - tdt * vy;
  }
  // :36-47
  void velForward() {
    #pragma omp parallel for schedule(static)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) {
        R ox, oy;
        if (i <= nx && j < ny) { trace(R(i), R(j) + R(0.5), dt, ox, oy); Uh[idxU(i, j)] = sU(U, ox, oy); }
        if (i < nx && j <= ny) { trace(R(i) + R(0.5), R(j), dt, ox, oy); Vh[idxV(i, j)] = sV(V, ox, oy); }
      }
  }
  // :49-66
  void velCorrect() {
    #pragma omp parallel for schedule(static)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) {
        R ox, oy, lo, hi;
        if (i <= nx && j < ny) {
          const int k = idxU(i, j); const R gx = R(i), gy = R(j) + R(0.5);
          trace(gx, gy, -dt, ox, oy); const R back = sU(Uh, ox, oy);
          trace(gx, gy, dt, ox, oy); mmU(U, ox, oy, lo, hi);
          U2[k] = clampv(Uh[k] + R(0.5) * (U[k] - back), lo, hi);
        }
        if (i < nx && j <= ny) {
          const int k = idxV(i, j); const R gx = R(i) + R(0.5), gy = R(j);
          trace(gx, gy, -dt, ox, oy); const R back = sV(Vh, ox, oy);
          trace(gx, gy, dt, ox, oy); mmV(V, ox, oy, lo, hi);
          V2[k] = clampv(Vh[k] + R(0.5) * (V[k] - back), lo, hi);
        }
      }
  }
  // :68-76
  void scalForward() {
    #pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const int k = idxC(i, j); R ox, oy;
        trace(R(i) + R(0.5), R(j) + R(0.5), dt, ox, oy);
        Th[k] = sC(T, Tamb, ox, oy);
        Yh[k] = sC4(Y, ox, oy);
      }
  }
  // :78-103
  void scalCorrect() {
    #pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const int k = idxC(i, j);
        const R gx = R(i) + R(0.5), gy = R(j) + R(0.5);
        R dxo, dyo, fxo, fyo; trace(gx, gy, dt, dxo, dyo); trace(gx, gy, -dt, fxo, fyo);
        R tlo, thi; mmC(T, Tamb, dxo, dyo, tlo, thi);
        Vec4<R> ylo, yhi; mmC4(Y, dxo, dyo, ylo, yhi);
        const R Tc = Th[k] + R(0.5) * (T[k] - sC(Th, Tamb, fxo, fyo));
        const Vec4<R> Yc = Yh[k] + R(0.5) * (Y[k] - sC4(Yh, fxo, fyo));
        const bool inT = Tc >= tlo && Tc <= thi;
        const bool inY = Yc.x >= ylo.x && Yc.y >= ylo.y && Yc.z >= ylo.z && Yc.w >= ylo.w &&
                         Yc.x <= yhi.x && Yc.y <= yhi.y && Yc.z <= yhi.z && Yc.w <= yhi.w;
        const R mixC = std::min(Yc.x, Yc.y / sO2);
        const R mixL = std::min(Yh[k].x, Yh[k].y / sO2);
        if (inT && inY && mixC <= mixL + R(1e-5)) { T2[k] = Tc; Y2[k] = Yc; }
        else { T2[k] = Th[k]; Y2[k] = Yh[k]; }
      }
  }

  // ---------------------------------------------------------------- diffuse.wgsl:18-50
  void diffuse(const std::vector<R>& Tin, const std::vector<Vec4<R>>& Yin, std::vector<R>& Tout, std::vector<Vec4<R>>& Yout) {
    const Vec4<R> mask{R(1), R(1), R(1), R(0)};
    #pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const int k = idxC(i, j);
        const R T0 = Tin[k]; const Vec4<R> Y0 = Yin[k];
        R sT = R(0); Vec4<R> sY{R(0), R(0), R(0), R(0)};
        auto face = [&](R f, int n) {
          if (f > R(0)) {
            const R a = f * rhoDOf(R(0.5) * (T0 + Tin[n]));
            sT += a * (Tin[n] - T0); sY = sY + a * (Yin[n] - Y0);
          }
        };
        if (i > 0) face(fx[idxU(i, j)], idxC(i - 1, j));
        if (i < nx - 1) face(fx[idxU(i + 1, j)], idxC(i + 1, j));
        if (j > 0) face(fy[idxV(i, j)], idxC(i, j - 1));
        if (j < ny - 1) face(fy[idxV(i, j + 1)], idxC(i, j + 1));
        const R c = diffDt / (rhoOf(T0) * dx * dx);
        Tout[k] = T0 + c * sT;
        Yout[k] = vmax(Y0 + (c * sY) * mask, Vec4<R>{R(0), R(0), R(0), R(0)});
      }
  }

  // ---------------------------------------------------------------- sources.wgsl:34-173
  std::vector<R> qrel_c, qrad_c, tpk_c;
  void sources() {
    const size_t nC = (size_t)nx * ny;
    qrel_c.assign(nC, R(0)); qrad_c.assign(nC, R(0)); tpk_c.assign(nC, R(0));
    const float E_SCALE = 1.0e6f, M_SCALE = 1.0e12f;
    #pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const int k = idxC(i, j);
        R qrel = R(0), qrad = R(0), tpeak = R(0);
        R Tc = T[k];
        Vec4<R> Yc = Y[k];
        const R sdf = gsdf[k];
        const uint32_t sid = gid[k];
        R massSrc = R(0);
        const R cellA = dx * dx;
        if (sdf < R(0) && sid != SOLID_NONE) {
          // :50-54 inside wood: hold the surface temperature
          const PieceF& pc = piece(sid >> 2u);
          T[k] = R(pc.Ts[sid & 3u]);
          SQ[k] = Vec2<R>{R(0), R(0)};
        } else {
          if (sid != SOLID_NONE && sdf < R(2) * dx) {          // :57-94 wood coupling
            const uint32_t pi = sid >> 2u, fi = sid & 3u;
            const PieceF& pc = piece(pi);
            const R Ts = R(pc.Ts[fi]);
            const R band = R(faceW[sid]) / R(1.0e8);
            const R w = std::max(R(0), R(1) - std::abs(sdf - dx) / dx) / dx * (R(2) * R(pc.half)) / std::max(band, R(1e-6));
            const R rho = rhoOf(Tc);
            const R kg = rhoDOf(R(0.5) * (Tc + Ts)) * cp;
            const R dist = std::max(sdf, R(0.5) * dx);
            const R rate = kg * w / (dist * rho * cp);
            const R dTc = (Ts - Tc) * (R(1) - std::exp(-rate * dt));
            Tc += dTc;
            const R toWood = -rho * cp * dTc * cellA;
            const int32_t q = wgsl_i32_round(toWood * R(E_SCALE));
            #pragma omp atomic
            acc[(pi * 4u + fi) * 2u] += q;
            const R mf = R(pc.mflux[fi]) * w;
            if (mf > R(0)) {
              const R madd = mf * dt;
              const R r = rhoOf(Tc);
              Yc = (r * Yc + Vec4<R>{madd, R(0), R(0), R(0)}) / (r + madd);
              Tc = (r * Tc + madd * Ts) / (r + madd);
              massSrc += mf;
            }
            const R cov = R(pc.charCov[fi]);
            if (cov > R(0) && Yc.y > R(0)) {
              const R r = rhoOf(Tc);
              const R kc = charA * std::exp(-charTa / Ts) * cov;
              const R mO2 = std::min(kc * r * Yc.y * w * dt, R(0.9) * r * Yc.y);
              const R mC = mO2 / charO2;
              Yc = (r * Yc + Vec4<R>{R(0), -mO2, mC + mO2, R(0)}) / (r + mC);
              Tc = (r * Tc + mC * Ts) / (r + mC);
              massSrc += mC / dt;
              const int32_t qm = wgsl_i32_round(mC * cellA * R(M_SCALE));
              #pragma omp atomic
              acc[(pi * 4u + fi) * 2u + 1u] += qm;
            }
          }
          // :96-107 test sources
          const R x = (R(i) + R(0.5)) * dx, y = (R(j) + R(0.5)) * dx;
          if (heaterT > R(0) && x > heaterX0 && x < heaterX1 && y < heaterY1) Tc = heaterT;
          if (burnerFlux > R(0) && j == 0 && x > burnerX0 && x < burnerX1) {
            const R mf = burnerFlux / dx;
            const R madd = mf * dt;
            const R r = rhoOf(Tc);
            Yc = (r * Yc + Vec4<R>{madd, R(0), R(0), R(0)}) / (r + madd);
            Tc = (r * Tc + madd * burnerT) / (r + madd);
            massSrc += mf;
          }
          // :109-120 gas-phase combustion, 8 sub-steps
          const R rho0 = rhoOf(Tc);
          const int NS = 8;
          const R h = dt / R(NS);
          R burned = R(0);
          for (int s = 0; s < NS; s++) {
            const R wr = reactB * rho0 * Yc.x * Yc.y * std::exp(-reactTa / Tc);
            const R dF = std::min(wr * h, std::min(Yc.x, Yc.y / sO2));
            Yc = Yc + Vec4<R>{-dF, -sO2 * dF, (R(1) + sO2) * dF, R(0)};
            Tc += dF * dHc / cp;
            burned += dF;
          }
          // :122-128 soot
          const R dSf = std::min(sootFormA * std::exp(-sootFormTa / Tc) * Yc.x * dt, Yc.x);
          Yc = Yc + Vec4<R>{-dSf, R(0), R(0), dSf};
          const R dSo = std::min(sootOxA * Yc.w * Yc.y * std::exp(-sootOxTa / Tc) * dt, std::min(Yc.w, Yc.y / sO2));
          Yc = Yc + Vec4<R>{R(0), -sO2 * dSo, (R(1) + sO2) * dSo, -dSo};
          Tc += dSo * dHc / cp;
          burned += dSo;
          qrel = rho0 * burned * dHc / dt;
          // :130-136 optically thin radiation, linearised implicit
          const R r1 = rhoOf(Tc);
          const R fv = r1 * Yc.w / sootDensity;
          const R kap = kappaSootC * fv * Tc + kappaGas * Yc.z;
          const R T3 = Tc * Tc * Tc;
          qrad = R(4) * kap * sigma * (T3 * Tc - std::pow(Tamb, R(4)));
          const R dTr = qrad * dt / (r1 * cp) / (R(1) + R(16) * kap * sigma * T3 * dt / (r1 * cp));
          Tc -= dTr;
          // :140-148 entrainment through the front/back faces
          const R ucx = R(0.5) * (U[idxU(i, j)] + U[idxU(i + 1, j)]);
          const R ucy = R(0.5) * (V[idxV(i, j)] + V[idxV(i, j + 1)]);
          const R me = R(2) * exchAlpha * std::sqrt(ucx * ucx + ucy * ucy) * rhoAmb / depth;
          if (me > R(0)) {
            const R madd = me * dt;
            const R r = rhoOf(Tc);
            Yc = (r * Yc + madd * ambY()) / (r + madd);
            Tc = (r * Tc + madd * Tamb) / (r + madd);
            massSrc += me;
          }
          // :150-156 write
          Tc = std::max(Tc, R(0.5) * Tamb);
          Yc = vmax(Yc, Vec4<R>{R(0), R(0), R(0), R(0)});
          const R S = massSrc / rhoOf(Tc) + std::log(Tc / T2[k]) / dt;
          T[k] = Tc; Y[k] = Yc; tpeak = Tc;
          SQ[k] = Vec2<R>{S, qrel};
        }
        qrel_c[k] = qrel; qrad_c[k] = qrad; tpk_c[k] = tpeak;
      }
    // :160-172 per-8x8-workgroup tree reduction, rounded to fixed point per workgroup
    const int gx = (nx + 7) / 8, gy = (ny + 7) / 8;
    const float G_SCALE = 1.0e3f;
    for (int wy = 0; wy < gy; wy++)
      for (int wxi = 0; wxi < gx; wxi++) {
        R rq[64], rr[64], rt[64];
        for (int li = 0; li < 64; li++) {
          const int i = wxi * 8 + (li & 7), j = wy * 8 + (li >> 3);
          const bool in = i < nx && j < ny;
          const R q = in ? qrel_c[idxC(i, j)] : R(0), r = in ? qrad_c[idxC(i, j)] : R(0);
          rq[li] = q * dx * dx * dt; rr[li] = r * dx * dx * dt; rt[li] = in ? tpk_c[idxC(i, j)] : R(0);
        }
        for (int s = 32; s > 0; s >>= 1)
          for (int li = 0; li < s; li++) { rq[li] += rq[li + s]; rr[li] += rr[li + s]; rt[li] = std::max(rt[li], rt[li + s]); }
        acc[ACC_GLOBAL] += wgsl_i32_round(rq[0] * R(G_SCALE));
        acc[ACC_GLOBAL + 1] += wgsl_i32_round(rr[0] * R(G_SCALE));
        acc[ACC_GLOBAL + 2] = std::max(acc[ACC_GLOBAL + 2], wgsl_i32((double)rt[0]));
      }
  }

  // ---------------------------------------------------------------- forces.wgsl:34-101
  R Tcl(int i, int j) const { return T[idxC(std::clamp(i, 0, nx - 1), std::clamp(j, 0, ny - 1))]; }
  R u2f(int i, int j) const { const int k = idxU(i, j); return fx[k] > R(0) ? U2[k] : R(0); }
  R v2f(int i, int j) const { const int k = idxV(i, j); return fy[k] > R(0) ? V2[k] : R(0); }
  R exchange(R spd, R Tf) const { return std::exp(R(-2.0) * exchAlpha * spd * (Tf / Tamb) / depth * dt); }
  void forces() {
    const R idx2 = R(1) / (dx * dx);
    #pragma omp parallel for schedule(static)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) {
        if (i <= nx && j < ny) {
          const int k = idxU(i, j);
          if (fx[k] <= R(0)) U[k] = R(0);
          else if (i == 0) U[k] = std::min(U2[idxU(1, j)], R(0));
          else if (i == nx) U[k] = std::max(U2[idxU(nx - 1, j)], R(0));
          else {
            const R u = U2[k];
            const R TL = Tcl(i - 1, j), TR = Tcl(i, j);
            const R rhoF = rhoOf(R(0.5) * (TL + TR));
            const R muE = muOf(TR), muW = muOf(TL);
            R uN = u, muN = muOf(R(0.5) * (TL + TR));
            if (j < ny - 1) { uN = u2f(i, j + 1); muN = muOf(R(0.25) * (TL + TR + Tcl(i - 1, j + 1) + Tcl(i, j + 1))); }
            R uS = -u, muS = muOf(R(0.5) * (TL + TR));
            if (j > 0) { uS = u2f(i, j - 1); muS = muOf(R(0.25) * (TL + TR + Tcl(i - 1, j - 1) + Tcl(i, j - 1))); }
            const R visc = (muE * (u2f(i + 1, j) - u) + muW * (u2f(i - 1, j) - u) + muN * (uN - u) + muS * (uS - u)) * idx2 / rhoF;
            const R vAvg = R(0.25) * (V2[idxV(i - 1, j)] + V2[idxV(i, j)] + V2[idxV(i - 1, j + 1)] + V2[idxV(i, j + 1)]);
            U[k] = (u + dt * visc) * exchange(std::sqrt(u * u + vAvg * vAvg), R(0.5) * (TL + TR));
          }
        }
        if (i < nx && j <= ny) {
          const int k = idxV(i, j);
          if (j == 0 || fy[k] <= R(0)) V[k] = R(0);
          else if (j == ny) V[k] = std::max(V2[idxV(i, ny - 1)], R(0));
          else {
            const R v = V2[k];
            const R TB = Tcl(i, j - 1), TT = Tcl(i, j);
            const R Tf = R(0.5) * (TB + TT);
            const R rhoF = rhoOf(Tf);
            const R muN = muOf(TT), muS = muOf(TB);
            R vE = v, muE = muOf(Tf);
            if (i < nx - 1) { vE = v2f(i + 1, j); muE = muOf(R(0.25) * (TB + TT + Tcl(i + 1, j - 1) + Tcl(i + 1, j))); }
            R vW = v, muW = muOf(Tf);
            if (i > 0) { vW = v2f(i - 1, j); muW = muOf(R(0.25) * (TB + TT + Tcl(i - 1, j - 1) + Tcl(i - 1, j))); }
            const R visc = (muN * (v2f(i, j + 1) - v) + muS * (v2f(i, j - 1) - v) + muE * (vE - v) + muW * (vW - v)) * idx2 / rhoF;
            const R buoy = grav * (Tf / Tamb - R(1));
            const R uAvg = R(0.25) * (U2[idxU(i, j - 1)] + U2[idxU(i + 1, j - 1)] + U2[idxU(i, j)] + U2[idxU(i + 1, j)]);
            V[k] = (v + dt * (visc + buoy)) * exchange(std::sqrt(uAvg * uAvg + v * v), Tf);
          }
        }
      }
  }

  // ---------------------------------------------------------------- pressure.wgsl
  R invRho(R t) const { return t / (rhoAmb * Tamb); }   // :27
  // :30-43
  void coef() {
    Level& L = lv[0];
    #pragma omp parallel for schedule(static)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) {
        if (i <= nx && j < ny) {
          const int k = idxU(i, j);
          const R Tf = R(0.5) * (T[idxC(std::clamp(i - 1, 0, nx - 1), j)] + T[idxC(std::min(i, nx - 1), j)]);
          L.ax[k] = fx[k] * invRho(Tf);
        }
        if (i < nx && j <= ny) {
          const int k = idxV(i, j);
          const R Tf = R(0.5) * (T[idxC(i, std::clamp(j - 1, 0, ny - 1))] + T[idxC(i, std::min(j, ny - 1))]);
          L.ay[k] = fy[k] * invRho(Tf);
        }
      }
  }
  // :46-54
  void rhs0() {
    Level& L = lv[0];
    #pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const R div = (fx[idxU(i + 1, j)] * U[idxU(i + 1, j)] - fx[idxU(i, j)] * U[idxU(i, j)]
                     + fy[idxV(i, j + 1)] * V[idxV(i, j + 1)] - fy[idxV(i, j)] * V[idxV(i, j)]) / dx;
        const R open = fx[idxU(i + 1, j)] + fx[idxU(i, j)] + fy[idxV(i, j + 1)] + fy[idxV(i, j)];
        L.rhs[idxC(i, j)] = open > R(0) ? (div - SQ[idxC(i, j)].x) / dt : R(0);
      }
  }
  // :57-67 (L = fine level l)
  void coefRestrict(int l) {
    const Level& F = lv[l]; Level& C = lv[l + 1];
    const int nxc = F.nx / 2, nyc = F.ny / 2;
    for (int J = 0; J <= nyc; J++)
      for (int I = 0; I <= nxc; I++) {
        if (I <= nxc && J < nyc)
          C.ax[J * (nxc + 1) + I] = R(0.5) * (F.ax[(2 * J) * (F.nx + 1) + 2 * I] + F.ax[(2 * J + 1) * (F.nx + 1) + 2 * I]);
        if (I < nxc && J <= nyc)
          C.ay[J * nxc + I] = R(0.5) * (F.ay[(2 * J) * F.nx + 2 * I] + F.ay[(2 * J) * F.nx + 2 * I + 1]);
      }
  }
  // :77-85 sum a*p_nb and diagonal (Dirichlet p = 0 at open faces: ghost = -p)
  static void stencil(const Level& L, const R* p, int i, int j, R& off, R& diag) {
    off = R(0); diag = R(0);
    const R w = L.ax[j * (L.nx + 1) + i], e = L.ax[j * (L.nx + 1) + i + 1];
    const R s = L.ay[j * L.nx + i], n = L.ay[(j + 1) * L.nx + i];
    if (i > 0) { off += w * p[j * L.nx + i - 1]; diag += w; } else { diag += R(2) * w; }
    if (i < L.nx - 1) { off += e * p[j * L.nx + i + 1]; diag += e; } else { diag += R(2) * e; }
    if (j > 0) { off += s * p[(j - 1) * L.nx + i]; diag += s; }
    if (j < L.ny - 1) { off += n * p[(j + 1) * L.nx + i]; diag += n; } else { diag += R(2) * n; }
  }
  // :87-94 (in place per colour: a colour pass reads only the other colour)
  void relax(int l, int color) {
    Level& L = lv[l];
    R* p = L.p.data();
    #pragma omp parallel for schedule(static)
    for (int j = 0; j < L.ny; j++)
      for (int i = (j + color) & 1; i < L.nx; i += 2) {
        R off, diag; stencil(L, p, i, j, off, diag);
        const int k = j * L.nx + i;
        p[k] = diag > R(0) ? (off - L.rhs[k] * L.h2) / diag : R(0);
      }
  }
  // :96-101
  R residual(const Level& L, int i, int j) const {
    R off, diag; stencil(L, L.p.data(), i, j, off, diag);
    const int k = j * L.nx + i;
    if (diag <= R(0)) return R(0);
    return L.rhs[k] - (off - diag * L.p[k]) / L.h2;
  }
  // :104-113
  void restrictRes(int l) {
    const Level& F = lv[l]; Level& C = lv[l + 1];
    const int nxc = F.nx / 2, nyc = F.ny / 2;
    #pragma omp parallel for schedule(static)
    for (int J = 0; J < nyc; J++)
      for (int I = 0; I < nxc; I++) {
        const R r = residual(F, 2 * I, 2 * J) + residual(F, 2 * I + 1, 2 * J) + residual(F, 2 * I, 2 * J + 1) + residual(F, 2 * I + 1, 2 * J + 1);
        C.rhs[J * nxc + I] = R(0.25) * r;
        C.p[J * nxc + I] = R(0);
      }
  }
  // :116-129
  void prolong(int l) {
    Level& F = lv[l]; const Level& C = lv[l + 1];
    const int nxc = F.nx / 2, nyc = F.ny / 2;
    #pragma omp parallel for schedule(static)
    for (int j = 0; j < F.ny; j++)
      for (int i = 0; i < F.nx; i++) {
        const int I = i / 2, J = j / 2;
        const int I2 = std::clamp(I + ((i & 1) == 1 ? 1 : -1), 0, nxc - 1);
        const int J2 = std::clamp(J + ((j & 1) == 1 ? 1 : -1), 0, nyc - 1);
        const R c = R(0.5625) * C.p[J * nxc + I] + R(0.1875) * (C.p[J * nxc + I2] + C.p[J2 * nxc + I]) + R(0.0625) * C.p[J2 * nxc + I2];
        const int k = j * F.nx + i;
        // only the diagonal of the stencil is used (closed cells get no correction)
        const R w = F.ax[j * (F.nx + 1) + i], e = F.ax[j * (F.nx + 1) + i + 1];
        const R s = F.ay[j * F.nx + i], n = F.ay[(j + 1) * F.nx + i];
        R diag = R(0);
        if (i > 0) diag += w; else diag += R(2) * w;
        if (i < F.nx - 1) diag += e; else diag += R(2) * e;
        if (j > 0) diag += s;
        if (j < F.ny - 1) diag += n; else diag += R(2) * n;
        F.p[k] += diag > R(0) ? c : R(0);
      }
  }
  // :132-156 (120 red-black sweeps from zero)
  void coarsest(int l) {
    Level& L = lv[l];
    const int n = L.nx * L.ny;
    std::vector<R> wp(n, R(0));
    for (int it = 0; it < 120; it++)
      for (int c = 0; c < 2; c++)
        for (int k = 0; k < n; k++) {
          const int i = k % L.nx, j = k / L.nx;
          if (((i + j) & 1) != c) continue;
          R off, diag; stencil(L, wp.data(), i, j, off, diag);
          wp[k] = diag > R(0) ? (off - L.rhs[k] * L.h2) / diag : R(0);
        }
    for (int k = 0; k < n; k++) L.p[k] = wp[k];
  }
  // Inverse of the coarsest operator in the library's operation order: A's lower
  // band (half-bandwidth nx, row-major cells; closed cells the row dmax e_k);
  // right-looking banded Cholesky (per column jc: L_jcjc = sqrt(a_jcjc), L_ijc =
  // a_ijc / L_jcjc, then a_ik = fma(-L_ijc, L_kjc, a_ik) for jc < k <= i <= jc+nx);
  // then column c of the inverse by forward and back substitution with the
  // reciprocal diagonal, k ascending. A pivot <= 1e-6 dmax (singular: a sealed gas
  // pocket) or a level wider than 32 cells leaves cinv_ok false.
  void coarse_factor() {
    const Level& L = lv.back();
    const int n = L.nx * L.ny, bw = L.nx, W = bw + 1;
    cinv_ok = false;
    if (n > 256 || bw > 32) return;
    std::vector<R> band((size_t)n * W, R(0)), dg(n), rinv(n);
    for (int k = 0; k < n; k++) {
      const int i = k % L.nx, j = k / L.nx;
      const R w = L.ax[j * (L.nx + 1) + i], e = L.ax[j * (L.nx + 1) + i + 1];
      const R so = L.ay[j * L.nx + i], no = L.ay[(j + 1) * L.nx + i];
      R diag = R(0);
      if (i > 0) diag += w; else diag += R(2) * w;
      if (i < L.nx - 1) diag += e; else diag += R(2) * e;
      if (j > 0) diag += so;
      if (j < L.ny - 1) diag += no; else diag += R(2) * no;
      dg[k] = diag;
      if (diag > R(0)) {
        band[(size_t)k * W] = diag;
        if (i > 0) band[(size_t)k * W + 1] = -w;
        if (j > 0) band[(size_t)k * W + bw] = -so;
      }
    }
    R dmax = R(0);
    for (int k = 0; k < n; k++) dmax = std::max(dmax, dg[k]);
    if (!(dmax > R(0))) return;
    const R thr = R(1e-6f) * dmax;
    for (int k = 0; k < n; k++)
      if (!(dg[k] > R(0))) band[(size_t)k * W] = dmax;
    auto B = [&](int i, int d) -> R& { return band[(size_t)i * W + d]; };
    std::vector<R> lij(bw);
    for (int jc = 0; jc < n; jc++) {
      const R piv = B(jc, 0);
      if (!(piv > thr)) return;
      const R ljj = std::sqrt(piv);
      for (int l = 0; l < bw; l++) {
        const int i = jc + 1 + l;
        if (i < n) lij[l] = B(i, i - jc) / ljj;
      }
      B(jc, 0) = ljj;
      for (int l = 0; l < bw; l++) {
        const int i = jc + 1 + l;
        if (i < n) B(i, i - jc) = lij[l];
      }
      for (int l = 0; l < bw; l++) {
        const int i = jc + 1 + l;
        if (i >= n) continue;
        for (int k = jc + 1; k <= i; k++) B(i, i - k) = std::fma(-lij[l], B(k, k - jc), B(i, i - k));
      }
    }
    for (int k = 0; k < n; k++) rinv[k] = R(1) / B(k, 0);
    std::vector<R> a((size_t)n * n), y(n);
    for (int c = 0; c < n; c++) {
      for (int i = 0; i < c; i++) y[i] = R(0);
      for (int i = c; i < n; i++) {
        R sum = i == c ? R(1) : R(0);
        for (int k = std::max(c, i - bw); k < i; k++) sum = std::fma(-B(i, i - k), y[k], sum);
        y[i] = sum * rinv[i];
      }
      for (int i = n - 1; i >= 0; i--) {
        R sum = y[i];
        const int kend = std::min(n - 1, i + bw);
        for (int k = i + 1; k <= kend; k++) sum = std::fma(-B(k, k - i), y[k], sum);
        y[i] = sum * rinv[i];
      }
      for (int i = 0; i < n; i++) a[(size_t)i * n + c] = y[i];
    }
    cinv = std::move(a);
    cinv_ok = true;
  }
  // p = A^-1 b, b = -rhs h2 (0 in closed cells); each row as 8 strided partial sums
  // (fma, increasing index) combined ((s0+s1)+(s2+s3))+((s4+s5)+(s6+s7))
  void coarsest_direct(int l) {
    Level& L = lv[l];
    const int n = L.nx * L.ny;
    std::vector<R> b(n);
    for (int k = 0; k < n; k++) {
      R off, diag; stencil(L, L.p.data(), k % L.nx, k / L.nx, off, diag);
      b[k] = diag > R(0) ? -(L.rhs[k] * L.h2) : R(0);
    }
    for (int k = 0; k < n; k++) {
      R sq[8];
      for (int q = 0; q < 8; q++) {
        sq[q] = R(0);
        for (int m = q; m < n; m += 8) sq[q] = std::fma(cinv[(size_t)k * n + m], b[m], sq[q]);
      }
      L.p[k] = ((sq[0] + sq[1]) + (sq[2] + sq[3])) + ((sq[4] + sq[5]) + (sq[6] + sq[7]));
    }
  }
  // js/fluid.js:294-312 (direct: the solve loop's cycles with the inverted coarsest level)
  void vcycle(int nu = 2, bool direct = false) {
    const int NL = (int)lv.size();
    for (int l = 0; l < NL - 1; l++) {
      for (int s = 0; s < nu; s++) { relax(l, 0); relax(l, 1); }
      restrictRes(l);
    }
    if (direct) coarsest_direct(NL - 1); else coarsest(NL - 1);
    for (int l = NL - 2; l >= 0; l--) {
      prolong(l);
      for (int s = 0; s < nu; s++) { relax(l, 1); relax(l, 0); }
    }
  }
  // The solve loop's cycle (extension of the library): the V-cycle above, or with w_cells > 0 the
  // W tail: the level two above the coarsest, if it has at most w_cells cells, visits the next
  // level twice per visit (the second visit smooths on from the first one's p; that level's rhs
  // is restricted once)
  void cycle_at(int l, bool direct) {
    const int NL = (int)lv.size();
    if (l == NL - 1) { if (direct) coarsest_direct(NL - 1); else coarsest(NL - 1); return; }
    for (int s = 0; s < 2; s++) { relax(l, 0); relax(l, 1); }
    restrictRes(l);
    const int g = (l == NL - 3 && (long)lv[l].nx * lv[l].ny <= w_cells) ? 2 : 1;
    for (int k = 0; k < g; k++) cycle_at(l + 1, direct);
    prolong(l);
    for (int s = 0; s < 2; s++) { relax(l, 1); relax(l, 0); }
  }
  void cycle(bool direct = false) {
    if (w_cells > 0) cycle_at(0, direct); else vcycle(2, direct);
  }
  // :159-180
  void project() {
    const std::vector<R>& p = lv[0].p;
    #pragma omp parallel for schedule(static)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) {
        if (i <= nx && j < ny) {
          const int k = idxU(i, j);
          if (fx[k] > R(0)) {
            const R pl = i > 0 ? p[idxC(std::max(i - 1, 0), j)] : -p[idxC(0, j)];
            const R pr = i < nx ? p[idxC(std::min(i, nx - 1), j)] : -p[idxC(nx - 1, j)];
            const R Tf = R(0.5) * (T[idxC(std::clamp(i - 1, 0, nx - 1), j)] + T[idxC(std::min(i, nx - 1), j)]);
            U[k] -= dt * invRho(Tf) * (pr - pl) / dx;
          } else U[k] = R(0);
        }
        if (i < nx && j <= ny) {
          const int k = idxV(i, j);
          if (j > 0 && fy[k] > R(0)) {
            const R pb = p[idxC(i, j - 1)];
            const R pt = j < ny ? p[idxC(i, std::min(j, ny - 1))] : -p[idxC(i, ny - 1)];
            const R Tf = R(0.5) * (T[idxC(i, j - 1)] + T[idxC(i, std::min(j, ny - 1))]);
            V[k] -= dt * invRho(Tf) * (pt - pb) / dx;
          } else V[k] = R(0);
        }
      }
  }

  // ---------------------------------------------------------------- pressure solve control (extension)
  // ||r||2 over level 0 with r from residual() (0 in closed cells), summed in FP64
  double res_norm() const {
    const Level& L = lv[0]; double s = 0;
    for (int j = 0; j < L.ny; j++) for (int i = 0; i < L.nx; i++) { const double r = (double)residual(L, i, j); s += r * r; }
    return std::sqrt(s);
  }
  double rhs_norm() const {
    double s = 0; for (const R v : lv[0].rhs) s += (double)v * (double)v; return std::sqrt(s);
  }
  // FP64 level-0 operator: r = rhs64 - A p64 with the f32 coefficients promoted
  double res64(std::vector<double>& r) const {
    const Level& L = lv[0]; const double h2 = (double)L.h2; double s = 0;
    r.assign((size_t)L.nx * L.ny, 0.0);
    for (int j = 0; j < L.ny; j++)
      for (int i = 0; i < L.nx; i++) {
        const double w = L.ax[j * (L.nx + 1) + i], e = L.ax[j * (L.nx + 1) + i + 1];
        const double so = L.ay[j * L.nx + i], n = L.ay[(j + 1) * L.nx + i];
        double off = 0, diag = 0;
        if (i > 0) { off += w * p64[j * L.nx + i - 1]; diag += w; } else diag += 2 * w;
        if (i < L.nx - 1) { off += e * p64[j * L.nx + i + 1]; diag += e; } else diag += 2 * e;
        if (j > 0) { off += so * p64[(j - 1) * L.nx + i]; diag += so; }
        if (j < L.ny - 1) { off += n * p64[(j + 1) * L.nx + i]; diag += n; } else diag += 2 * n;
        const int k = j * L.nx + i;
        const double rv = diag > 0 ? rhs64[k] - (off - diag * p64[k]) / h2 : 0.0;
        r[k] = rv; s += rv * rv;
      }
    return std::sqrt(s);
  }
  // q = L d at level 0 in FP64: (sum a d_nb - diag d) / h2 (0 in closed cells)
  void lap64(const std::vector<double>& d, std::vector<double>& q) const {
    const Level& L = lv[0]; const double h2 = (double)L.h2;
    q.assign((size_t)L.nx * L.ny, 0.0);
    for (int j = 0; j < L.ny; j++)
      for (int i = 0; i < L.nx; i++) {
        const double w = L.ax[j * (L.nx + 1) + i], e = L.ax[j * (L.nx + 1) + i + 1];
        const double so = L.ay[j * L.nx + i], n = L.ay[(j + 1) * L.nx + i];
        double off = 0, diag = 0;
        if (i > 0) { off += w * d[j * L.nx + i - 1]; diag += w; } else diag += 2 * w;
        if (i < L.nx - 1) { off += e * d[j * L.nx + i + 1]; diag += e; } else diag += 2 * e;
        if (j > 0) { off += so * d[(j - 1) * L.nx + i]; diag += so; }
        if (j < L.ny - 1) { off += n * d[(j + 1) * L.nx + i]; diag += n; } else diag += 2 * n;
        const int k = j * L.nx + i;
        q[k] = diag > 0 ? (off - diag * d[k]) / h2 : 0.0;
      }
  }
  // FP64 mode, Krylov variant: flexible (Polak-Ribiere) preconditioned CG on the level-0
  // operator, one FP32 V-cycle on f32(r) per iteration as the preconditioner z ~ L^-1 r:
  // delta = r.z; beta = -alpha_prev (q_prev.z) / delta_prev; d = z + beta d; q = L d kept
  // as Lz + beta q (L symmetric), with d.q = z.Lz + 2 beta (q_prev.z) + beta^2 (d.q)_prev;
  // alpha = delta / (d.q); p64 += alpha d; r -= alpha q; stop on ||r|| / ||rhs64|| with
  // ||r - alpha q||^2 = r.r - 2 alpha (r.Lz + beta r.q_prev) + alpha^2 (Lz.Lz + 2 beta
  // Lz.q_prev + beta^2 q_prev.q_prev) from the dot products taken before the update (the
  // GPU's fused Krylov mode decides from these before it updates r).
  void pressure_pcg(bool direct) {
    rhs0_64();
    double b = 0; for (double v : rhs64) b += v * v; b = std::sqrt(b);
    std::vector<double> r, z, d, q, lz;
    double rn = res64(r);
    last_rel0 = b > 0 ? rn / b : 0.0;
    Level& L0 = lv[0];
    const size_t n = r.size();
    d.assign(n, 0.0); q.assign(n, 0.0); z.assign(n, 0.0);
    double alpha = 0, delta_prev = 0, pi_prev = 0;
    int c = 0;
    while (b > 0 && rn / b > tol && c < max_cycles) {
      for (size_t k = 0; k < n; k++) { L0.rhs[k] = R((float)r[k]); L0.p[k] = R(0); }
      cycle(direct);
      for (size_t k = 0; k < n; k++) z[k] = (double)L0.p[k];
      lap64(z, lz);
      // delta = r.z, eta = q.z, zeta = z.Lz; beta (Polak-Ribiere); d.q = zeta + 2 beta eta +
      // beta^2 (d.q)_prev with d = z + beta d and q = Lz + beta q (L symmetric); alpha = delta / d.q
      double delta = 0, eta = 0, zeta = 0, rr = 0, rl = 0, rq = 0, ll = 0, lq = 0, qq = 0;
      for (size_t k = 0; k < n; k++) {
        delta += r[k] * z[k]; eta += q[k] * z[k]; zeta += z[k] * lz[k];
        rr += r[k] * r[k]; rl += r[k] * lz[k]; rq += r[k] * q[k]; ll += lz[k] * lz[k]; lq += lz[k] * q[k]; qq += q[k] * q[k];
      }
      const bool more = c > 0 && delta_prev != 0;
      const double beta = more ? -alpha * eta / delta_prev : 0.0;
      const double pi = more ? zeta + 2.0 * beta * eta + beta * beta * pi_prev : zeta;
      alpha = pi != 0 ? delta / pi : 0.0;
      delta_prev = delta; pi_prev = pi;
      const double rqc = rl + beta * rq, qqc = ll + 2.0 * beta * lq + beta * beta * qq;
      const double s2 = rr - 2.0 * alpha * rqc + alpha * alpha * qqc;
      for (size_t k = 0; k < n; k++) {
        d[k] = c == 0 ? z[k] : z[k] + beta * d[k];
        q[k] = c == 0 ? lz[k] : lz[k] + beta * q[k];
        p64[k] += alpha * d[k];
        r[k] -= alpha * q[k];
      }
      c++;
      rn = std::sqrt(s2 > 0 ? s2 : 0.0);
    }
    last_cycles = c; last_rel = b > 0 ? rn / b : 0.0;
  }
  // FP64 divergence-source assembly (the FP64 counterpart of rhs0)
  void rhs0_64() {
    const double ddx = (double)dx, ddt = (double)dt;
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const double a = (double)fx[idxU(i + 1, j)] * (double)U[idxU(i + 1, j)], b = (double)fx[idxU(i, j)] * (double)U[idxU(i, j)];
        const double c = (double)fy[idxV(i, j + 1)] * (double)V[idxV(i, j + 1)], d = (double)fy[idxV(i, j)] * (double)V[idxV(i, j)];
        const double open = (double)fx[idxU(i + 1, j)] + (double)fx[idxU(i, j)] + (double)fy[idxV(i, j + 1)] + (double)fy[idxV(i, j)];
        rhs64[idxC(i, j)] = open > 0 ? (((a - b) + c - d) / ddx - (double)SQ[idxC(i, j)].x) / ddt : 0.0;
      }
  }
  void project64() {
    const double ddt = (double)dt, ddx = (double)dx, rT = (double)(rhoAmb * Tamb);
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) {
        if (i <= nx && j < ny) {
          const int k = idxU(i, j);
          if (fx[k] > R(0)) {
            const double pl = i > 0 ? p64[idxC(i - 1, j)] : -p64[idxC(0, j)];
            const double pr = i < nx ? p64[idxC(std::min(i, nx - 1), j)] : -p64[idxC(nx - 1, j)];
            const double Tf = 0.5 * ((double)T[idxC(std::clamp(i - 1, 0, nx - 1), j)] + (double)T[idxC(std::min(i, nx - 1), j)]);
            U[k] = R((double)U[k] - ddt * (Tf / rT) * (pr - pl) / ddx);
          } else U[k] = R(0);
        }
        if (i < nx && j <= ny) {
          const int k = idxV(i, j);
          if (j > 0 && fy[k] > R(0)) {
            const double pb = p64[idxC(i, j - 1)];
            const double pt = j < ny ? p64[idxC(i, std::min(j, ny - 1))] : -p64[idxC(i, ny - 1)];
            const double Tf = 0.5 * ((double)T[idxC(i, j - 1)] + (double)T[idxC(i, std::min(j, ny - 1))]);
            V[k] = R((double)V[k] - ddt * (Tf / rT) * (pt - pb) / ddx);
          } else V[k] = R(0);
        }
      }
  }
  // coarse_direct 2 (pipelined): the cycles use the inverse factored during the previous
  // step; this step's operator is factored after its solve for the next step
  void pressure_solve() {
    pressure_solve_inner();
    if (coarse_direct == 2 && mode != SOLVE_FIXED) coarse_factor();
  }
  void pressure_solve_inner() {
    if (mode == SOLVE_FIXED) {
      for (int c = 0; c < ncycles; c++) cycle();
      last_cycles = ncycles;
      const double b = rhs_norm(); last_rel = b > 0 ? res_norm() / b : 0.0;
      return;
    }
    if (coarse_direct == 1) coarse_factor();
    const bool direct = coarse_direct && cinv_ok;
    if (mode == SOLVE_TOL) {
      const double b = rhs_norm();
      int c = 0; double rel = 0;
      do { cycle(direct); c++; rel = b > 0 ? res_norm() / b : 0.0; } while (rel > tol && c < max_cycles);
      last_cycles = c; last_rel = rel;
      return;
    }
    if (krylov) { pressure_pcg(direct); return; }
    // SOLVE_FP64: FP32 V-cycles on the defect inside an FP64 loop
    rhs0_64();
    double b = 0; for (double v : rhs64) b += v * v; b = std::sqrt(b);
    std::vector<double> r;
    double rn = res64(r);
    last_rel0 = b > 0 ? rn / b : 0.0;
    int c = 0;
    Level& L0 = lv[0];
    while (b > 0 && rn / b > tol && c < max_cycles) {
      for (size_t k = 0; k < r.size(); k++) { L0.rhs[k] = R((float)r[k]); L0.p[k] = R(0); }
      cycle(direct); c++;
      for (size_t k = 0; k < r.size(); k++) p64[k] += (double)L0.p[k];
      rn = res64(r);
    }
    last_cycles = c; last_rel = b > 0 ? rn / b : 0.0;
  }

  // ---------------------------------------------------------------- geometry.wgsl
  void nearest(R px, R py, R& best, uint32_t& bid) const {   // :121-130
    best = R(1e9); bid = SOLID_NONE;
    for (int n = 0; n < P.nPieces; n++) {
      const PieceF& pc = piece(n);
      if (pc.alive <= 0.0f) continue;
      const R d = sdBox(px, py, pc);
      if (d < best) { best = d; bid = (uint32_t)n * 4u + faceOf(px, py, pc); }
    }
  }
  void clear_geometry() { std::memset(faceW, 0, sizeof faceW); }   // js/fluid.js:213
  void geometry() {                                                // :132-153
    const float W_SCALE = 1.0e8f;
    #pragma omp parallel for schedule(static)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) {
        if (i < nx && j < ny) {
          R best; uint32_t bid;
          nearest((R(i) + R(0.5)) * dx, (R(j) + R(0.5)) * dx, best, bid);
          gsdf[idxC(i, j)] = best; gid[idxC(i, j)] = bid;
          if (bid != SOLID_NONE && best >= R(0) && best < R(2) * dx) {
            const R w = std::max(R(0), R(1) - std::abs(best - dx) / dx) / dx;
            const int32_t q = wgsl_i32_round(w * dx * dx * R(W_SCALE));
            #pragma omp atomic
            faceW[bid] += q;
          }
        }
        if (i <= nx && j < ny) {
          R d; uint32_t b; nearest(R(i) * dx, (R(j) + R(0.5)) * dx, d, b);
          fx[idxU(i, j)] = clampv(R(0.5) + d / dx, R(0), R(1));
        }
        if (i < nx && j <= ny) {
          R d; uint32_t b; nearest((R(i) + R(0.5)) * dx, R(j) * dx, d, b);
          fy[idxV(i, j)] = j == 0 ? R(0) : clampv(R(0.5) + d / dx, R(0), R(1));
        }
      }
  }

  // ---------------------------------------------------------------- radiation.wgsl
  static R planck580(R t) {   // :28-33
    const R l = R(580e-9);
    const R x = R(1.438777e-2) / (l * t);
    if (x > R(80)) return R(0);
    return R(1.191042e-16) / (l * l * l * l * l) / (std::exp(x) - R(1)) * R(1e-9);
  }
  // :36-51 ray vs rotated box: (t_enter, face) or t < 0
  void hitBox(R ox, R oy, R dxr, R dyr, const PieceF& pc, R& tn_out, R& face) const {
    const R c = std::cos(R(pc.angle)), s = std::sin(R(pc.angle));
    const R qx = ox - R(pc.pos[0]), qy = oy - R(pc.pos[1]);
    const R lox = c * qx + s * qy, loy = -s * qx + c * qy;
    const R ldx = c * dxr + s * dyr, ldy = -s * dxr + c * dyr;
    const R h = R(pc.half);
    const R invx = R(1) / (std::abs(ldx) < R(1e-9) ? R(1e-9) : ldx);
    const R invy = R(1) / (std::abs(ldy) < R(1e-9) ? R(1e-9) : ldy);
    const R t1x = (-h - lox) * invx, t1y = (-h - loy) * invy;
    const R t2x = (h - lox) * invx, t2y = (h - loy) * invy;
    const R tminx = std::min(t1x, t2x), tminy = std::min(t1y, t2y);
    const R tmaxx = std::max(t1x, t2x), tmaxy = std::max(t1y, t2y);
    const R tn = std::max(tminx, tminy), tf = std::min(tmaxx, tmaxy);
    if (tf < R(0) || tn > tf || tn < R(1e-5)) { tn_out = R(-1); face = R(0); return; }
    if (tminx > tminy) face = ldx < R(0) ? R(0) : R(2); else face = ldy < R(0) ? R(1) : R(3);
    tn_out = tn;
  }
  // :53-62
  void gasAt(R px, R py, R& gx, R& gy) const {
    const int i = wgsl_i32((double)(px / dx)), j = wgsl_i32((double)(py / dx));
    if (i < 0 || j < 0 || i >= nx || j >= ny) { gx = R(0); gy = R(0); return; }
    const int k = idxC(i, j);
    const R Tg = T[k]; const Vec4<R> Yg = Y[k];
    const R fv = rhoOf(Tg) * Yg.w / sootDensity;
    const R kap = kappaSootC * fv * Tg + kappaGas * Yg.z;
    const R T2v = Tg * Tg;
    gx = kap * sigma * (T2v * T2v - std::pow(Tamb, R(4))) / R(3.14159265);
    gy = R(6.3) * fv / R(580e-9) * planck580(Tg);
  }
  // :64-158 (one workgroup of NRAY rays per face or floor probe)
  void radiation() {
    const R PI = R(3.14159265);
    const int NRAY = nray;
    const uint32_t nFaces = (uint32_t)P.nPieces * 4u;
    const int ntgt = P.nPieces * 4 + N_FLOOR;
    #pragma omp parallel for schedule(dynamic)
    for (int tg = 0; tg < ntgt; tg++) {
      const uint32_t tgt = (uint32_t)tg;
      std::vector<R> sq(NRAY), sv(NRAY);
      bool valid_wg = false;
      for (int li = 0; li < NRAY; li++) {
        R ox0 = 0, oy0 = 0, nrx = 0, nry = 1; bool valid = false;
        if (tgt < nFaces) {
          const PieceF& pc = piece(tgt / 4u);
          const uint32_t f = tgt % 4u;
          if (pc.alive > 0.0f) {
            const R c = std::cos(R(pc.angle)), s = std::sin(R(pc.angle));
            R lnx = 1, lny = 0;
            if (f == 1u) { lnx = 0; lny = 1; } else if (f == 2u) { lnx = -1; lny = 0; } else if (f == 3u) { lnx = 0; lny = -1; }
            nrx = c * lnx - s * lny; nry = s * lnx + c * lny;
            const R tx = -nry, ty = nrx;
            const R u = (fract(R(li) * R(0.618034) + R(P.frame) * R(0.1234)) - R(0.5)) * R(1.6) * R(pc.half);
            const R hh = R(pc.half) + R(1e-4);
            ox0 = R(pc.pos[0]) + nrx * hh + tx * u; oy0 = R(pc.pos[1]) + nry * hh + ty * u;
            valid = true;
          }
        } else {
          const uint32_t fi = tgt - nFaces;
          if (fi < (uint32_t)N_FLOOR) {
            ox0 = (R(fi) + R(0.5)) / R(N_FLOOR) * R(P.nx) * dx; oy0 = R(1e-4);
            nrx = 0; nry = 1; valid = true;
          }
        }
        valid_wg = valid;
        R dq = 0, dv = 0;
        if (valid) {
          const R jit = fract(R(P.frame) * R(0.7548777) + R(tgt) * R(0.5698403));
          const R a = ((R(li) + jit) / R(NRAY) - R(0.5)) * PI;
          const R cosn = std::cos(a);
          const R base = std::atan2(nry, nrx);
          R ddx = std::cos(base + a), ddy = std::sin(base + a);
          R ox = ox0, oy = oy0;
          R J = 0, Jv = 0, Twall = Tamb;
          bool bounced = false;
          const R ds = dx;
          for (int step = 0; step < 4096; step++) {
            R tHit = R(1e9), hitT = R(0);
            for (int n = 0; n < P.nPieces; n++) {
              const PieceF& pc = piece(n);
              if (pc.alive <= 0.0f) continue;
              R hx, hy; hitBox(ox, oy, ddx, ddy, pc, hx, hy);
              if (hx > R(0) && hx < tHit) { tHit = hx; hitT = R(pc.Ts[(uint32_t)hy]); }
            }
            R tFloor = R(1e9);
            if (ddy < R(-1e-6)) tFloor = -oy / ddy;
            const R tEnd = std::min(tHit, tFloor);
            const R W = R(P.nx) * dx, H = R(P.ny) * dx;
            R tx = R(1e9), ty = R(1e9);
            if (ddx > R(1e-6)) tx = (W - ox) / ddx; else if (ddx < R(-1e-6)) tx = -ox / ddx;
            if (ddy > R(1e-6)) ty = (H - oy) / ddy;
            const R tOut = std::min(std::min(tx, ty), tEnd);
            const int ns = wgsl_i32((double)std::ceil(tOut / ds));
            for (int m = 0; m < ns; m++) {
              const R t = (R(m) + R(0.5)) * tOut / R(ns);
              R gx, gy; gasAt(ox + ddx * t, oy + ddy * t, gx, gy);
              J += gx * tOut / R(ns);
              Jv += gy * tOut / R(ns);
            }
            if (tHit < tFloor && tHit < R(1e8)) { Twall = hitT; break; }
            if (tFloor < R(1e8) && tFloor <= tHit && !bounced) {
              ox = ox + ddx * tFloor; oy = oy + ddy * tFloor + R(1e-5);
              ddy = -ddy;
              bounced = true;
              continue;
            }
            Twall = Tamb;
            break;
          }
          const R w = PI / R(NRAY) * cosn;
          const R T2v = Twall * Twall;
          dq = w * (R(0.5) * sigma * T2v * T2v + R(2) * J);
          dv = w * (R(2) * Jv);
        }
        sq[li] = dq; sv[li] = dv;
      }
      for (int s = NRAY / 2; s > 0; s >>= 1)
        for (int li = 0; li < s; li++) { sq[li] += sq[li + s]; sv[li] += sv[li + s]; }
      if (valid_wg) {
        float* o = &rad[tgt * 4];
        const R oldq = R(o[0]), oldv = R(o[1]);
        const R a = oldq <= R(0) ? R(1) : R(0.35);
        o[0] = (float)mix(oldq, sq[0], a); o[1] = (float)mix(oldv, sv[0], a); o[2] = 0; o[3] = 0;
      }
    }
  }

  // ---------------------------------------------------------------- step (js/fluid.js:225-253)
  void stage_advect() { scalForward(); scalCorrect(); velForward(); velCorrect(); }
  void stage_diffuse() {
    diffuse(T2, Y2, T, Y);
    for (int s = 1; s < diffSub; s += 2) { diffuse(T, Y, Th, Yh); diffuse(Th, Yh, T, Y); }
  }
  void stage_coef_rhs() {
    coef(); rhs0();
    for (int l = 0; l < (int)lv.size() - 1; l++) coefRestrict(l);
  }
  void stage_project() {
    if (mode == SOLVE_FP64) project64(); else project();
  }
  void step() {
    stage_advect();
    stage_diffuse();
    sources();
    forces();
    stage_coef_rhs();
    pressure_solve();
    stage_project();
    time += dtd;
    if (cfl > 0) update_dt();
  }
  // CFL step for the next step (extension): dt = min(dt_cap, cfl * dx / max|u|), then
  // the diffusion sub-step count of js/fluid.js:190-198 for the new dt.
  double max_speed() const {
    float m = 0.f;
    for (const R v : U) m = std::max(m, std::abs((float)v));
    for (const R v : V) m = std::max(m, std::abs((float)v));
    return m;
  }
  void update_dt() {
    const float m = (float)max_speed();
    const float cand = m > 0.f ? (float)cfl * P.dx / m : (float)dt_cap;
    dtd = (double)std::min((float)dt_cap, cand);
    host.dt = (float)dtd;
    write_params();
  }

  // js/fluid.js:315-324 + afterSubmit: copy out and clear acc
  void readback(int32_t* acc_out, float* rad_out, int32_t* faceW_out) {
    if (acc_out) std::memcpy(acc_out, acc, sizeof acc);
    if (rad_out) std::memcpy(rad_out, rad, sizeof rad);
    if (faceW_out) std::memcpy(faceW_out, faceW, sizeof faceW);
    std::memset(acc, 0, sizeof acc);
  }

  // FP64 budgets over the gas cells (extension): mass, energy, species masses per m depth
  void budgets(double* out) const {
    double m = 0, e = 0, mf = 0, mo = 0, mp = 0, ms = 0, q = 0, tmax = 0;
    const double cellA = (double)dx * (double)dx;
    for (int k = 0; k < nx * ny; k++) {
      if (gsdf[k] < R(0) && gid[k] != SOLID_NONE) continue;
      const double t = (double)T[k];
      const double rho = (double)rhoAmb * (double)Tamb / t;
      m += rho * cellA; e += rho * (double)cp * t * cellA;
      mf += rho * (double)Y[k].x * cellA; mo += rho * (double)Y[k].y * cellA;
      mp += rho * (double)Y[k].z * cellA; ms += rho * (double)Y[k].w * cellA;
      q += (double)SQ[k].y * cellA; tmax = std::max(tmax, t);
    }
    out[0] = m; out[1] = e; out[2] = mf; out[3] = mo; out[4] = mp; out[5] = ms; out[6] = q; out[7] = tmax;
  }
};

}  // namespace cforc
