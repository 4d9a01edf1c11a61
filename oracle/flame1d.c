/* ORACLE — test infrastructure, not product code.
 *
 * FP64 1D freely propagating premixed flame with the gas model of campfire's
 * simulator, restated from tests/flame1d.mjs:1-71 (BoccheseGiacomo/campfire):
 * rho ~ 1/T, Sutherland mu(T) (:10), unity Lewis number, cp = 1300, one-step
 * Arrhenius F + s O2 -> (1+s) P with the caps of :41-43, continuity du/dx = S
 * (:48), first-order upwind advection (:50-58) and front tracking at T > 1200 K
 * (:61). The flame speed is S_L = lab speed * Tu / Tb (:66-70).
 *
 * Known answer (README.md:89, js/config.js:26): B = 2e10, Ta = 15000 K,
 * resolved (dx = 5e-5, L = 0.03, tEnd = 1) gives S_L = 0.38 m/s.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double kTamb = 293.15, kRhoAmb = 1.2, kCp = 1300, kPr = 0.7, kDHc = 15e6, kYO = 0.232;
#define SO2 (15e6 / 13.1e6)

static double mu_of(double T) { return 1.716e-5 * pow(T / 273.15, 1.5) * 383.55 / (T + 110.4); }

/* returns S_L (0 when the front never crosses 30% .. 75% of the domain); *Tb_out = peak T */
double flame1d_speed(double B, double Ta, double dx, double F, double phi, double L, double tEnd, double* Tb_out) {
  const int n = (int)lround(L / dx);
  const double YFst = kYO / SO2;
  const double YF0 = phi * YFst / (1 + phi * YFst) * 1, YO0 = kYO / (1 + phi * YFst);
  double *T = malloc(sizeof(double) * n), *YF = malloc(sizeof(double) * n), *YO = malloc(sizeof(double) * n);
  double *Tn = malloc(sizeof(double) * n), *Fn = malloc(sizeof(double) * n), *On = malloc(sizeof(double) * n);
  double *S = malloc(sizeof(double) * n), *u = calloc((size_t)n + 1, sizeof(double));
  for (int i = 0; i < n; i++) { T[i] = kTamb; YF[i] = YF0; YO[i] = YO0; }
  const int nign = (int)lround(0.01 / dx);
  for (int i = 0; i < nign && i < n; i++) { T[i] = 2000; YF[i] = 0; YO[i] = fmax(0, YO0 - SO2 * YF0); }
  const double alphaMax = mu_of(2300) / kPr * F / (kRhoAmb * kTamb / 2300);
  const double dt = fmin(0.2 * dx * dx / alphaMax, 0.2 * dx / 6);
  double t = 0, Tb = 0;
  /* front track: first sample past 30% and past 75% of L, else the last sample */
  double ta = -1, xa = 0, tbk = -1, xb = 0, tlast = 0, xlast = 0;
  while (t < tEnd) {
    memcpy(Tn, T, sizeof(double) * n); memcpy(Fn, YF, sizeof(double) * n); memcpy(On, YO, sizeof(double) * n);
    for (int i = 0; i < n; i++) {
      const double rho = kRhoAmb * kTamb / T[i];
      double dT = 0, dF = 0, dO = 0;
      for (int s = 0; s < 2; s++) {
        const int j = s == 0 ? i - 1 : i + 1;
        if (j < 0 || j >= n) continue;
        const double a = mu_of(0.5 * (T[i] + T[j])) / kPr * F;
        dT += a * (T[j] - T[i]); dF += a * (YF[j] - YF[i]); dO += a * (YO[j] - YO[i]);
      }
      const double c = dt / (rho * dx * dx);
      Tn[i] += c * dT; Fn[i] += c * dF; On[i] += c * dO;
      const double w = B * rho * Fn[i] * On[i] * exp(-Ta / Tn[i]) / F;
      const double d = fmin(fmin(w * dt, Fn[i]), On[i] / SO2);
      Fn[i] -= d; On[i] -= SO2 * d; Tn[i] += d * kDHc / kCp;
      S[i] = log(Tn[i] / T[i]) / dt;
    }
    memcpy(T, Tn, sizeof(double) * n); memcpy(YF, Fn, sizeof(double) * n); memcpy(YO, On, sizeof(double) * n);
    for (int i = 0; i < n; i++) u[i + 1] = u[i] + S[i] * dx;
    for (int i = 0; i < n; i++) {
      const double uc = 0.5 * (u[i] + u[i + 1]);
      const int j = uc > 0 ? i - 1 : i + 1;
      const int k = j < 0 ? 0 : (j > n - 1 ? n - 1 : j);
      const double cfl = fabs(uc) * dt / dx;
      Tn[i] = T[i] + cfl * (T[k] - T[i]); Fn[i] = YF[i] + cfl * (YF[k] - YF[i]); On[i] = YO[i] + cfl * (YO[k] - YO[i]);
    }
    memcpy(T, Tn, sizeof(double) * n); memcpy(YF, Fn, sizeof(double) * n); memcpy(YO, On, sizeof(double) * n);
    t += dt;
    double xf = 0;
    for (int i = 0; i < n; i++) if (T[i] > 1200) xf = (i + 0.5) * dx;
    for (int i = 0; i < n; i++) Tb = fmax(Tb, T[i]);
    if (ta < 0 && xf > 0.3 * L) { ta = t; xa = xf; }
    if (tbk < 0 && xf > 0.75 * L) { tbk = t; xb = xf; }
    tlast = t; xlast = xf;
    if (xf > L * 0.8) break;
  }
  free(T); free(YF); free(YO); free(Tn); free(Fn); free(On); free(S); free(u);
  if (Tb_out) *Tb_out = Tb;
  if (tbk < 0) { tbk = tlast; xb = xlast; }
  if (ta < 0 || tbk <= ta) return 0;
  return (xb - xa) / (tbk - ta) * kTamb / Tb;
}
