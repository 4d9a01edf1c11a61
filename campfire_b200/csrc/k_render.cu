// Headless renderer: shaders/render.wgsl's fragment stage (fs, :189-273, with
// the colour science :52-141, the wood cross-section :143-181 and floorVis
// :183-188) as one CUDA thread per pixel writing linear RGBA floats (the
// fragment output, before the swapchain's 8-bit quantisation) into a device
// image whose row 0 is the top of the picture. The vertex stage's full-screen
// triangle is replaced by the pixel centre: uv = ((x + 0.5) / W, 1 - (y + 0.5) / H).
// Every expression keeps render.wgsl's operation order (the library is built
// with -fmad=false); WGSL abstract-float constants are the nearest f32.
#include "gas_dev.cuh"
#include "kernels.h"

namespace cfg {

namespace {

struct V3 { float x, y, z; };
__device__ __forceinline__ V3 v3(float a) { return {a, a, a}; }
__device__ __forceinline__ V3 v3(float a, float b, float c) { return {a, b, c}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ V3 vmax(V3 a, V3 b) { return {a.x < b.x ? b.x : a.x, a.y < b.y ? b.y : a.y, a.z < b.z ? b.z : a.z}; }
__device__ __forceinline__ V3 vmin(V3 a, V3 b) { return {b.x < a.x ? b.x : a.x, b.y < a.y ? b.y : a.y, b.z < a.z ? b.z : a.z}; }
__device__ __forceinline__ V3 vclamp(V3 e, float lo, float hi) { return vmin(vmax(e, v3(lo)), v3(hi)); }
__device__ __forceinline__ float fmin_w(float a, float b) { return b < a ? b : a; }   // WGSL min
__device__ __forceinline__ float fmax_w(float a, float b) { return a < b ? b : a; }   // WGSL max
__device__ __forceinline__ float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 mix3(V3 a, V3 b, float t) { return {mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)}; }
__device__ __forceinline__ float fract_w(float x) { return x - floorf(x); }
// smoothstep(low, high, x) = t * t * (3 - 2 t), t = clamp((x - low) / (high - low), 0, 1)
__device__ __forceinline__ float smooth_w(float lo, float hi, float x) {
  const float t = fmin_w(fmax_w((x - lo) / (hi - lo), 0.f), 1.f);
  return t * t * (3.f - 2.f * t);
}

// :53-56
__device__ __forceinline__ float g3(float x, float mu, float s1, float s2) {
  const float t = (x - mu) / (x < mu ? s1 : s2);
  return expf(-0.5f * t * t);
}
// :58-63 CIE 1931 2-degree matching functions (Wyman, Sloan & Shirley 2013 fit)
__device__ __forceinline__ V3 cie(float l) {
  const float x = 1.056f * g3(l, 599.8f, 37.9f, 31.0f) + 0.362f * g3(l, 442.0f, 16.0f, 26.7f) -
                  0.065f * g3(l, 501.1f, 20.4f, 26.2f);
  const float y = 0.821f * g3(l, 568.8f, 46.9f, 40.5f) + 0.286f * g3(l, 530.9f, 16.3f, 31.1f);
  const float z = 1.217f * g3(l, 437.0f, 11.8f, 36.0f) + 0.681f * g3(l, 459.0f, 26.0f, 13.8f);
  return {x, y, z};
}
// :64-69
__device__ __forceinline__ V3 xyz2rgb(V3 c) {
  return {3.2406f * c.x - 1.5372f * c.y - 0.4986f * c.z, -0.9689f * c.x + 1.8758f * c.y + 0.0415f * c.z,
          0.0557f * c.x - 0.2040f * c.y + 1.0570f * c.z};
}
// :71-76 Planck spectral radiance, W/(m^2 sr nm)
__device__ __forceinline__ float planck(float lnm, float T) {
  const float l = lnm * 1e-9f;
  const float x = 1.438777e-2f / (l * T);
  if (x > 80.0f) return 0.f;
  return 1.191042e-16f / (l * l * l * l * l) / (expf(x) - 1.0f) * 1e-9f;
}
// :81
__device__ __forceinline__ float spline(float l, float l0, float w) {
  const float t = (l - l0) / w;
  return expf(-0.5f * t * t) / (2.5066f * w);
}
constexpr int NL = 12;
__device__ __forceinline__ float lam(int n) { return 400.0f + ((float)n + 0.5f) * 300.0f / (float)NL; }

struct RenderIn {
  const SceneDesc* S;
  cfg_render_params R;
  const float4* wood;   // MAX_PIECES x (Tp, d, misc)
};

// :86-96
__device__ V3 gasXYZ(const RenderIn& in, float Tg, float fv, float q) {
  const cfg_params& P = in.S->P;
  V3 xyz = v3(0.f);
  for (int n = 0; n < NL; n++) {
    const float l = lam(n);
    const float k = 6.3f * fv / (l * 1e-9f);
    float L = (1.0f - expf(-k * P.depth)) * planck(l, Tg);
    L += in.R.chemi * q * P.depth / 12.566f * (0.6f * spline(l, 431.0f, 6.0f) + 0.4f * spline(l, 516.0f, 8.0f));
    xyz = xyz + cie(l) * L;
  }
  return xyz * (300.0f / (float)NL);
}
// :97-102
__device__ V3 greyXYZ(float Ts, float eps) {
  if (Ts < 650.0f) return v3(0.f);
  V3 xyz = v3(0.f);
  for (int n = 0; n < NL; n++) {
    const float l = lam(n);
    xyz = xyz + cie(l) * eps * planck(l, Ts);
  }
  return xyz * (300.0f / (float)NL);
}
// :104-109
__device__ V3 fireLightXYZ() {
  V3 xyz = v3(0.f);
  const float b0 = planck(580.0f, 1400.0f) / 580.0f;
  for (int n = 0; n < NL; n++) {
    const float l = lam(n);
    xyz = xyz + cie(l) * planck(l, 1400.0f) / l / b0;
  }
  return xyz * (300.0f / (float)NL);
}
// :110-113
__device__ __forceinline__ float srgb1(float s) {
  return s <= 0.0031308f ? 12.92f * s : 1.055f * powf(s, (float)(1.0 / 2.4)) - 0.055f;
}
__device__ __forceinline__ V3 srgbEncode(V3 c) {
  const V3 s = vclamp(c, 0.f, 1.f);
  return {srgb1(s.x), srgb1(s.y), srgb1(s.z)};
}
// :117-132
__device__ V3 tonemapXYZ(const RenderIn& in, V3 xyz, V3 base) {
  const float L = fmax_w(xyz.y * in.R.exposure, 0.f);
  const float L0 = 0.001f, Lw = 20.0f;
  const float Ld = logf(1.0f + L / L0) / logf(1.0f + Lw / L0);
  V3 rgb = v3(0.f);
  if (xyz.y > 1e-12f) {
    const V3 c = vmax(xyz2rgb(xyz / xyz.y), v3(0.f));
    const float lum = dot3(c, v3(0.2126f, 0.7152f, 0.0722f));
    const V3 pre = c / fmax_w(lum, 1e-6f) * powf(Ld, 2.2f) * 1.6f;
    rgb = {1.0f - expf(-pre.x), 1.0f - expf(-pre.y), 1.0f - expf(-pre.z)};
  }
  return srgbEncode(rgb + base);
}
// :133-140
__device__ V3 inferno(float t0) {
  const float t = fmin_w(fmax_w(t0, 0.f), 1.f);
  const V3 c0 = v3(0.0002f, 0.0016f, -0.0194f), c1 = v3(0.1065f, 0.5640f, 3.9327f);
  const V3 c2 = v3(11.6024f, -3.9728f, -15.9423f), c3 = v3(-41.7040f, 17.4364f, 44.3541f);
  const V3 c4 = v3(77.1629f, -33.4023f, -81.8073f), c5 = v3(-71.3194f, 32.6261f, 73.2095f);
  const V3 c6 = v3(25.1311f, -12.2426f, -23.0703f);
  return vclamp(c0 + t * (c1 + t * (c2 + t * (c3 + t * (c4 + t * (c5 + t * c6))))), 0.f, 1.f);
}
// :141-145
__device__ __forceinline__ float hash2(float px, float py) { return fract_w(sinf(px * 127.1f + py * 311.7f) * 43758.5453f); }
__device__ float vnoise(float px, float py) {
  const float ix = floorf(px), iy = floorf(py), fx = fract_w(px), fy = fract_w(py);
  const float ux = fx * fx * (3.0f - 2.0f * fx), uy = fy * fy * (3.0f - 2.0f * fy);
  return mixf(mixf(hash2(ix, iy), hash2(ix + 1.0f, iy + 0.0f), ux), mixf(hash2(ix + 0.0f, iy + 1.0f), hash2(ix + 1.0f, iy + 1.0f), ux),
              uy);
}

// :148-159
struct WoodHit { int idx; float lx, ly; };
__device__ WoodHit woodAt(const RenderIn& in, float px, float py) {
  const Piece* pcs = reinterpret_cast<const Piece*>(in.S->pieces);
  for (int n = in.R.nPieces - 1; n >= 0; n--) {
    const Piece pc = pcs[n];
    if (pc.alive <= 0.0f) continue;
    const float c = cosf(pc.angle), s = sinf(pc.angle);
    const float qx = px - pc.pos[0], qy = py - pc.pos[1];
    const float lx = c * qx + s * qy, ly = -s * qx + c * qy;
    if (fabsf(lx) <= pc.half && fabsf(ly) <= pc.half) return {n, lx, ly};
  }
  return {-1, 0.f, 0.f};
}
// :164-181
struct WoodPix { float T, ch; };
__device__ WoodPix woodProfile(const Piece& pc, const float4* w, float lx, float ly) {
  const float h = pc.half;
  const float dep[4] = {h - lx, h - ly, h + lx, h + ly};
  const float m = fmin_w(fmin_w(dep[0], dep[1]), fmin_w(dep[2], dep[3]));
  const float Tp[4] = {w[0].x, w[0].y, w[0].z, w[0].w}, dd4[4] = {w[1].x, w[1].y, w[1].z, w[1].w};
  const float4 misc = w[2];
  float T = 0.f, ch = 0.f, ws = 0.f;
  #pragma unroll
  for (int f = 0; f < 4; f++) {
    const float wgt = expf(-(dep[f] - m) / (0.15f * h));
    const float dd = dep[f];
    const float cd = fmax_w(dd4[f], 1e-5f);
    float Tf;
    if (dd < cd) Tf = mixf(pc.Ts[f], Tp[f], dd / cd);
    else Tf = mixf(Tp[f], misc.y, smooth_w(cd, h, dd));
    T += wgt * Tf;
    ch += wgt * ((dd < cd || misc.w < 0.5f) ? 1.0f : 0.0f);
    ws += wgt;
  }
  return {T / ws, ch / ws};
}
// :183-188
__device__ float floorVis(const RenderIn& in, float x) {
  const int base = in.R.nPieces * 4;
  const float fx = fmin_w(fmax_w(x / in.R.width * (float)N_FLOOR - 0.5f, 0.0f), (float)(N_FLOOR - 1));
  const int i0 = wgsl_i32(floorf(fx)), i1 = min(i0 + 1, N_FLOOR - 1);
  return mixf(in.S->rad[base + i0].y, in.S->rad[base + i1].y, fx - floorf(fx));
}
// :25-29 sQ: the heat-release sampler
__device__ __forceinline__ float fQ(const SceneDesc& S, int i, int j) {
  if (i < 0 || i >= S.nx || j < 0 || j >= S.ny) return 0.f;
  return S.SQ[j * S.pc + i].y;
}
__device__ float sQ(const SceneDesc& S, float gx, float gy) {
  const float fx = gx - 0.5f, fy = gy - 0.5f;
  const float bx = floorf(fx), by = floorf(fy), tx = fx - bx, ty = fy - by;
  const int i = wgsl_i32(bx), j = wgsl_i32(by);
  return mixf(mixf(fQ(S, i, j), fQ(S, i + 1, j), tx), mixf(fQ(S, i, j + 1), fQ(S, i + 1, j + 1), tx), ty);
}

// :189-273
__device__ float4 fragment(const RenderIn& in, float uvx, float uvy) {
  const SceneDesc& S = *in.S;
  const cfg_params& P = S.P;
  const cfg_render_params& R = in.R;
  const float wx = uvx * R.width / R.zoom + R.camX, wy = uvy * (R.height + R.ground) / R.zoom + R.camY;
  const float gx = wx / P.dx, gy = wy / P.dx;
  const WoodHit hit = woodAt(in, wx, wy);
  const bool ground = wy < 0.0f;
  const CField sT{S.T, S.nx, S.ny, S.pc, P.Tamb};
  const C4Field sY{S.Y, S.nx, S.ny, S.pc, ambY(P)};
  const Piece* pcs = reinterpret_cast<const Piece*>(S.pieces);

  if (R.view == 0) {
    V3 xyz = v3(0.f), rgbAdd = v3(0.f);
    const V3 fl = fireLightXYZ();
    if (hit.idx >= 0) {
      const Piece pc = pcs[hit.idx];
      const float4* w = in.wood + 3 * hit.idx;
      const WoodPix wp = woodProfile(pc, w, hit.lx, hit.ly);
      const float r = sqrtf(hit.lx * hit.lx + hit.ly * hit.ly) / pc.half;
      const float rings =
          0.5f + 0.5f * sinf(r * 38.0f + vnoise(hit.lx * 300.0f, hit.ly * 300.0f) * 2.0f + (float)hit.idx * 3.0f);
      const V3 grain = v3(0.42f, 0.28f, 0.15f) * (0.8f + 0.25f * rings) *
                       (0.85f + 0.3f * vnoise(hit.lx * 900.0f, hit.ly * 900.0f));
      const float o13 = (float)hit.idx * 13.0f;
      const float crackN = vnoise(hit.lx * 420.0f + o13, hit.ly * 420.0f + o13);
      const float crack = smooth_w(0.72f, 0.8f, crackN);
      const V3 charCol = v3(0.035f, 0.032f, 0.03f) * (0.7f + 0.6f * vnoise(hit.lx * 1500.0f, hit.ly * 1500.0f));
      const V3 albedo = mix3(grain, charCol, wp.ch);
      const float Tglow = wp.T * (1.0f + 0.05f * crack * wp.ch);
      xyz = xyz + greyXYZ(Tglow, 0.9f);
      xyz = xyz + fl * dot3(albedo, v3(0.2126f, 0.7152f, 0.0722f)) * w[2].z * 0.035f / 3.14159f;
      rgbAdd = albedo * 0.006f;
    } else if (ground) {
      const float n = vnoise(wx * 180.0f, wy * 180.0f) * 0.6f + vnoise(wx * 900.0f, wy * 900.0f) * 0.4f;
      const V3 alb = v3(0.16f, 0.13f, 0.10f) * (0.6f + 0.6f * n);
      const float fade = expf(wy / R.ground * 2.5f);
      xyz = xyz + fl * floorVis(in, wx) / 3.14159f * dot3(alb, v3(0.333f)) * fade * 0.06f;
      rgbAdd = alb * 0.01f;
    } else {
      const float Tg = sample(sT, gx, gy, 0.5f, 0.5f);
      const float4 Yg = sample4(sY, gx, gy);
      const float rho = rhoOf(P, Tg);
      const float fv = rho * Yg.w / P.sootDensity;
      xyz = xyz + gasXYZ(in, Tg, fv, sQ(S, gx, gy));
      rgbAdd = mix3(v3(0.006f, 0.006f, 0.010f), v3(0.0015f, 0.0015f, 0.003f), uvy);
    }
    const V3 c = tonemapXYZ(in, xyz, rgbAdd);
    return make_float4(c.x, c.y, c.z, 1.0f);
  }

  V3 col = v3(0.f);
  if (R.view == 1) {
    float Tv = P.Tamb;
    if (hit.idx >= 0) Tv = woodProfile(pcs[hit.idx], in.wood + 3 * hit.idx, hit.lx, hit.ly).T;
    else if (!ground) Tv = sample(sT, gx, gy, 0.5f, 0.5f);
    col = inferno((Tv - P.Tamb) / (R.tmax - P.Tamb));
    if (ground) col = v3(0.08f);
  } else if (!ground && hit.idx < 0) {
    const float4 Yg = sample4(sY, gx, gy);
    if (R.view == 2) {
      col = inferno(powf(sQ(S, gx, gy) / 2.0e7f, 0.5f));
    } else if (R.view == 3) {
      col = mix3(v3(0.02f, 0.02f, 0.08f), v3(0.35f, 0.85f, 1.0f), Yg.y / fmax_w(P.YOamb, 1e-3f));
    } else if (R.view == 4) {
      col = inferno(sqrtf(Yg.x / 0.4f));
    } else if (R.view == 5) {
      const int gix = wgsl_i32(gx), giy = wgsl_i32(gy);
      const int ii = min(max(gix, 0), S.nx - 1), jj = min(max(giy, 0), S.ny - 1);
      const float u = 0.5f * (S.U[jj * S.pu + ii] + S.U[jj * S.pu + ii + 1]);
      const float v = 0.5f * (S.V[jj * S.pc + ii] + S.V[(jj + 1) * S.pc + ii]);
      col = inferno(sqrtf(u * u + v * v) / 3.0f);
    } else if (R.view == 6) {
      col = inferno(sqrtf(rhoOf(P, sample(sT, gx, gy, 0.5f, 0.5f)) * Yg.w / P.sootDensity / 1e-6f));
    }
  } else if (ground) {
    col = v3(0.08f);
  } else {
    col = v3(0.35f, 0.3f, 0.25f);
  }
  // piece outlines
  if (hit.idx >= 0) {
    const float h = pcs[hit.idx].half;
    const float e = h - fmax_w(fabsf(hit.lx), fabsf(hit.ly));
    col = mix3(col, v3(0.85f), (1.0f - smooth_w(0.0f, 0.0012f, e)) * 0.6f);
  }
  return make_float4(col.x, col.y, col.z, 1.0f);
}

}  // namespace

__global__ void __launch_bounds__(256) k_render(const SceneDesc* __restrict__ scenes, int scene, cfg_render_params R,
                                                const float4* __restrict__ wood, int W, int H, float4* __restrict__ out) {
  const int x = blockIdx.x * 16 + (threadIdx.x & 15), y = blockIdx.y * 16 + (threadIdx.x >> 4);
  if (x >= W || y >= H) return;
  const RenderIn in{scenes + scene, R, wood};
  const float uvx = ((float)x + 0.5f) / (float)W, uvy = 1.0f - ((float)y + 0.5f) / (float)H;
  out[(size_t)y * W + x] = fragment(in, uvx, uvy);
}

void launch_render(const SceneDesc* scenes, int scene, const cfg_render_params& R, const float* wood, int W, int H,
                   float* out, cudaStream_t st) {
  const dim3 grid((W + 15) / 16, (H + 15) / 16);
  k_render<<<grid, 256, 0, st>>>(scenes, scene, R, reinterpret_cast<const float4*>(wood), W, H,
                                 reinterpret_cast<float4*>(out));
}

}  // namespace cfg
