/*
 * emc_oracle.c -- CPU restatement of emClarity's orientation-search hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library and
 * the timed CPU baseline; the product never links or calls it.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 *
 * The same source is compiled twice (see oracle/Makefile):
 *   REAL = double -> liboracle_f64.so, the FP64 oracle the GPU path is checked against;
 *   REAL = float  -> liboracle_f32.so, a single-precision port of the reference CPU
 *                    path (MATLAB single: interpn + fftn + BH_multi_xcf_*), used as the
 *                    timed CPU baseline with OpenMP over orientations.
 *
 * Every function cites the reference file:line it restates (paths relative to the
 * emClarity source tree).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef REAL
#define REAL double
#endif
#ifndef SFX
#define SFX _f64
#endif
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

#define EXPORT __attribute__((visibility("default")))

typedef struct { REAL re, im; } cplx;

static inline cplx c_mul(cplx a, cplx b) { cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static inline cplx c_add(cplx a, cplx b) { cplx r = {a.re + b.re, a.im + b.im}; return r; }
static inline cplx c_sub(cplx a, cplx b) { cplx r = {a.re - b.re, a.im - b.im}; return r; }

/* ------------------------------------------------------------------ rotation matrix */
/* BH_defineMatrix(ANGLES,'Bah',DIRECTION) -- coordinates/BH_defineMatrix.m:85-126.
 * R = Rz(a3) Rx(a2) Rz(a1) after negating ('forward') or reversing ('inv') the angles.
 * Output column-major like MATLAB. */
EXPORT void FN(orc_define_matrix)(const double ang_deg[3], int direction, double R[9]) {
  double a[3];
  for (int i = 0; i < 3; ++i) a[i] = ang_deg[i] * (M_PI / 180.0);
  if (direction == 0) { /* forward: angles = -angles (:85-86) */
    for (int i = 0; i < 3; ++i) a[i] = -a[i];
  } else { /* inv: angles = flip(angles) (:87-102) */
    double t = a[0]; a[0] = a[2]; a[2] = t;
  }
  double c[3], s[3];
  for (int i = 0; i < 3; ++i) { c[i] = cos(a[i]); s[i] = sin(a[i]); }
  double Z3[9] = {c[2], s[2], 0, -s[2], c[2], 0, 0, 0, 1};   /* column-major */
  double X2[9] = {1, 0, 0, 0, c[1], s[1], 0, -s[1], c[1]};
  double Z1[9] = {c[0], s[0], 0, -s[0], c[0], 0, 0, 0, 1};
  double T[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double acc = 0;
      for (int k = 0; k < 3; ++k) acc += Z3[i + 3 * k] * X2[k + 3 * j];
      T[i + 3 * j] = acc;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double acc = 0;
      for (int k = 0; k < 3; ++k) acc += T[i + 3 * k] * Z1[k + 3 * j];
      R[i + 3 * j] = acc;
    }
}

/* ------------------------------------------------------------------ interpolation */
static inline REAL vox(const REAL* v, int nx, int ny, int nz, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return 0;
  return v[((long)z * ny + y) * nx + x];
}

/* trilinear, interpn(...,'linear',0) (transformations/BH_resample3d.m:242): 0 outside [0,n-1] */
static REAL interp_linear(const REAL* v, int nx, int ny, int nz, double sx, double sy, double sz, int border) {
  if (!border) {
    if (sx < 0 || sy < 0 || sz < 0 || sx > nx - 1 || sy > ny - 1 || sz > nz - 1) return 0;
  } else {
    /* texture border addressing: zero-valued voxels around the volume (mexXform3d.cu:269-271) */
    if (sx <= -1 || sy <= -1 || sz <= -1 || sx >= nx || sy >= ny || sz >= nz) return 0;
  }
  int x0 = (int)floor(sx), y0 = (int)floor(sy), z0 = (int)floor(sz);
  double fx = sx - x0, fy = sy - y0, fz = sz - z0;
  double acc = 0;
  for (int dz = 0; dz < 2; ++dz)
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) {
        double w = (dx ? fx : 1 - fx) * (dy ? fy : 1 - fy) * (dz ? fz : 1 - fz);
        if (w == 0) continue;
        acc += w * (double)vox(v, nx, ny, nz, x0 + dx, y0 + dy, z0 + dz);
      }
  return (REAL)acc;
}

/* Catmull-Rom cubic convolution weights for the four taps at offsets -1..2 */
static inline void cr_weights(double t, double w[4]) {
  double t2 = t * t, t3 = t2 * t;
  w[0] = 0.5 * (-t3 + 2 * t2 - t);
  w[1] = 0.5 * (3 * t3 - 5 * t2 + 2);
  w[2] = 0.5 * (-3 * t3 + 4 * t2 + t);
  w[3] = 0.5 * (t3 - t2);
}

/* tricubic (Catmull-Rom) with zero-valued voxels outside; 0 outside [0,n-1] */
static REAL interp_cubic(const REAL* v, int nx, int ny, int nz, double sx, double sy, double sz) {
  if (sx < 0 || sy < 0 || sz < 0 || sx > nx - 1 || sy > ny - 1 || sz > nz - 1) return 0;
  int x0 = (int)floor(sx), y0 = (int)floor(sy), z0 = (int)floor(sz);
  double wx[4], wy[4], wz[4];
  cr_weights(sx - x0, wx);
  cr_weights(sy - y0, wy);
  cr_weights(sz - z0, wz);
  double acc = 0;
  for (int k = 0; k < 4; ++k)
    for (int j = 0; j < 4; ++j) {
      double wyz = wy[j] * wz[k];
      for (int i = 0; i < 4; ++i)
        acc += wx[i] * wyz * (double)vox(v, nx, ny, nz, x0 - 1 + i, y0 - 1 + j, z0 - 1 + k);
    }
  return (REAL)acc;
}

/* derivative of the Catmull-Rom weights w.r.t. t */
static inline void cr_dweights(double t, double w[4]) {
  double t2 = t * t;
  w[0] = 0.5 * (-3 * t2 + 4 * t - 1);
  w[1] = 0.5 * (9 * t2 - 10 * t);
  w[2] = 0.5 * (-9 * t2 + 8 * t + 1);
  w[3] = 0.5 * (3 * t2 - 2 * t);
}

/* value and gradient of the tricubic interpolant (for the adjoint oracle) */
static double interp_cubic_grad(const REAL* v, int nx, int ny, int nz, double sx, double sy, double sz,
                                double g[3]) {
  g[0] = g[1] = g[2] = 0;
  if (sx < 0 || sy < 0 || sz < 0 || sx > nx - 1 || sy > ny - 1 || sz > nz - 1) return 0;
  int x0 = (int)floor(sx), y0 = (int)floor(sy), z0 = (int)floor(sz);
  double wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
  cr_weights(sx - x0, wx); cr_dweights(sx - x0, dx);
  cr_weights(sy - y0, wy); cr_dweights(sy - y0, dy);
  cr_weights(sz - z0, wz); cr_dweights(sz - z0, dz);
  double acc = 0;
  for (int k = 0; k < 4; ++k)
    for (int j = 0; j < 4; ++j)
      for (int i = 0; i < 4; ++i) {
        double val = (double)vox(v, nx, ny, nz, x0 - 1 + i, y0 - 1 + j, z0 - 1 + k);
        acc += wx[i] * wy[j] * wz[k] * val;
        g[0] += dx[i] * wy[j] * wz[k] * val;
        g[1] += wx[i] * dy[j] * wz[k] * val;
        g[2] += wx[i] * wy[j] * dz[k] * val;
      }
  return acc;
}

/* value and gradient of the trilinear interpolant (interpn semantics, 0 outside [0,n-1]) */
static double interp_linear_grad(const REAL* v, int nx, int ny, int nz, double sx, double sy, double sz,
                                 double g[3]) {
  g[0] = g[1] = g[2] = 0;
  if (sx < 0 || sy < 0 || sz < 0 || sx > nx - 1 || sy > ny - 1 || sz > nz - 1) return 0;
  const int x0 = (int)floor(sx), y0 = (int)floor(sy), z0 = (int)floor(sz);
  const double fx = sx - x0, fy = sy - y0, fz = sz - z0;
  double c[2][2][2];
  for (int dz = 0; dz < 2; ++dz)
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) c[dz][dy][dx] = (double)vox(v, nx, ny, nz, x0 + dx, y0 + dy, z0 + dz);
  double val = 0;
  for (int dz = 0; dz < 2; ++dz)
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) {
        const double wx = dx ? fx : 1 - fx, wy = dy ? fy : 1 - fy, wz = dz ? fz : 1 - fz;
        val += wx * wy * wz * c[dz][dy][dx];
        g[0] += (dx ? 1.0 : -1.0) * wy * wz * c[dz][dy][dx];
        g[1] += wx * (dy ? 1.0 : -1.0) * wz * c[dz][dy][dx];
        g[2] += wx * wy * (dz ? 1.0 : -1.0) * c[dz][dy][dx];
      }
  return val;
}

/* Sample position of output voxel p (mexXform3d.cu:45-65 with the texture-coordinate
 * shift of :293-296 and :67-74 folded back to index space, i.e. s = M u + floor(n/2)):
 *   fwd : u = p - c - shift ; s = M u + c
 *   inv : u = p - c         ; s = M u + shift + c                                   */
static inline void sample_pos(const double M[9], const double sh[3], int fwd, int x, int y, int z, int cx, int cy,
                              int cz, double s[3]) {
  double u[3] = {(double)(x - cx), (double)(y - cy), (double)(z - cz)};
  if (fwd) { u[0] -= sh[0]; u[1] -= sh[1]; u[2] -= sh[2]; }
  for (int i = 0; i < 3; ++i) s[i] = M[i] * u[0] + M[i + 3] * u[1] + M[i + 6] * u[2];
  if (!fwd) { s[0] += sh[0]; s[1] += sh[1]; s[2] += sh[2]; }
  s[0] += cx; s[1] += cy; s[2] += cz;
}

/* mexXform3d / interpolator.interp3d (testScripts/interpolator.m:99-154): average over
 * nsym matrices.  interp: 0 linear (interpn), 1 cubic, 2 linear with zero border. */
EXPORT void FN(orc_rotate)(const REAL* src, int nx, int ny, int nz, const double* M, int nsym, const double sh[3],
                           int fwd, int interp, REAL* out) {
  const int cx = nx / 2, cy = ny / 2, cz = nz / 2;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        double acc = 0;
        for (int k = 0; k < nsym; ++k) {
          double s[3];
          sample_pos(M + 9 * k, sh, fwd, x, y, z, cx, cy, cz, s);
          acc += interp == 1 ? interp_cubic(src, nx, ny, nz, s[0], s[1], s[2])
                             : interp_linear(src, nx, ny, nz, s[0], s[1], s[2], interp == 2);
        }
        out[((long)z * ny + y) * nx + x] = (REAL)(acc / nsym);
      }
}

/* ------------------------------------------------------------------ FFT */
/* Own mixed-radix FFT (Stockham autosort; radices 4, 2, 3, 5 and a direct DFT for any
 * other prime factor).  Stands in for MATLAB fftn / cuFFT, which compute the same DFT. */
typedef struct {
  int n;
  int nf;
  int f[32];
  cplx* tw; /* exp(-2 pi i m/n) */
} fftplan;

static void plan_init(fftplan* p, int n) {
  p->n = n;
  p->nf = 0;
  int m = n;
  while (m % 4 == 0) { p->f[p->nf++] = 4; m /= 4; }
  while (m % 2 == 0) { p->f[p->nf++] = 2; m /= 2; }
  while (m % 3 == 0) { p->f[p->nf++] = 3; m /= 3; }
  while (m % 5 == 0) { p->f[p->nf++] = 5; m /= 5; }
  for (int q = 7; m > 1; q += 2)
    while (m % q == 0) { p->f[p->nf++] = q; m /= q; }
  p->tw = (cplx*)malloc(sizeof(cplx) * (n > 0 ? n : 1));
  for (int k = 0; k < n; ++k) {
    double a = -2.0 * M_PI * (double)k / (double)n;
    p->tw[k].re = (REAL)cos(a);
    p->tw[k].im = (REAL)sin(a);
  }
}
static void plan_free(fftplan* p) { free(p->tw); }

/* in-place complex FFT of x (length p->n) using work buffer w; sign -1 forward, +1 inverse */
static void fft1(const fftplan* p, cplx* x, cplx* w, int sign) {
  const int n = p->n;
  if (n == 1) return;
  cplx* src = x;
  cplx* dst = w;
  int ns = 1;
  for (int s = 0; s < p->nf; ++s) {
    const int R = p->f[s];
    const int nb = n / R;
    cplx v[64];
    for (int j = 0; j < nb; ++j) {
      const int k = j % ns;
      for (int r = 0; r < R; ++r) {
        cplx a = src[j + r * nb];
        if (ns > 1 && r) {
          cplx t = p->tw[((long)r * k * (n / (ns * R))) % n];
          if (sign > 0) t.im = -t.im;
          a = c_mul(a, t);
        }
        v[r] = a;
      }
      cplx o[64];
      if (R == 2) {
        o[0] = c_add(v[0], v[1]); o[1] = c_sub(v[0], v[1]);
      } else if (R == 4) {
        cplx a0 = c_add(v[0], v[2]), a1 = c_sub(v[0], v[2]);
        cplx b0 = c_add(v[1], v[3]), d = c_sub(v[1], v[3]);
        cplx b1 = sign < 0 ? (cplx){d.im, -d.re} : (cplx){-d.im, d.re};
        o[0] = c_add(a0, b0); o[2] = c_sub(a0, b0); o[1] = c_add(a1, b1); o[3] = c_sub(a1, b1);
      } else {
        for (int q = 0; q < R; ++q) {
          cplx acc = {0, 0};
          for (int r = 0; r < R; ++r) {
            double a = sign * 2.0 * M_PI * (double)((long)q * r % R) / (double)R;
            cplx t = {(REAL)cos(a), (REAL)sin(a)};
            acc = c_add(acc, c_mul(v[r], t));
          }
          o[q] = acc;
        }
      }
      const int idx = (j / ns) * ns * R + k;
      for (int r = 0; r < R; ++r) dst[idx + r * ns] = o[r];
    }
    cplx* t = src; src = dst; dst = t;
    ns *= R;
  }
  if (src != x) memcpy(x, src, sizeof(cplx) * n);
}

/* 3-D R2C, unnormalised, half spectrum (nx/2+1)*ny*nz in FFT order (mexFFT.cu:205-218) */
EXPORT void FN(orc_fft3_r2c)(const REAL* in, int nx, int ny, int nz, REAL* out_c) {
  const int nxh = nx / 2 + 1;
  cplx* out = (cplx*)out_c;
  fftplan px, py, pz;
  plan_init(&px, nx); plan_init(&py, ny); plan_init(&pz, nz);
  int mx = nx > ny ? nx : ny; mx = mx > nz ? mx : nz;
  cplx* line = (cplx*)malloc(sizeof(cplx) * mx);
  cplx* work = (cplx*)malloc(sizeof(cplx) * mx);
  for (long r = 0; r < (long)ny * nz; ++r) {
    for (int x = 0; x < nx; ++x) { line[x].re = in[r * nx + x]; line[x].im = 0; }
    fft1(&px, line, work, -1);
    for (int k = 0; k < nxh; ++k) out[r * nxh + k] = line[k];
  }
  for (int z = 0; z < nz; ++z)
    for (int k = 0; k < nxh; ++k) {
      for (int y = 0; y < ny; ++y) line[y] = out[((long)z * ny + y) * nxh + k];
      fft1(&py, line, work, -1);
      for (int y = 0; y < ny; ++y) out[((long)z * ny + y) * nxh + k] = line[y];
    }
  for (int y = 0; y < ny; ++y)
    for (int k = 0; k < nxh; ++k) {
      for (int z = 0; z < nz; ++z) line[z] = out[((long)z * ny + y) * nxh + k];
      fft1(&pz, line, work, -1);
      for (int z = 0; z < nz; ++z) out[((long)z * ny + y) * nxh + k] = line[z];
    }
  free(line); free(work);
  plan_free(&px); plan_free(&py); plan_free(&pz);
}

/* 3-D C2R, unnormalised (cufftExecC2R, mexFFT.cu:223); imaginary parts of the kx=0 and
 * kx=nx/2 terms are ignored, i.e. the real part of the Hermitian inverse. */
EXPORT void FN(orc_fft3_c2r)(const REAL* in_c, int nx, int ny, int nz, REAL* out) {
  const int nxh = nx / 2 + 1;
  const long nh = (long)nxh * ny * nz;
  cplx* tmp = (cplx*)malloc(sizeof(cplx) * nh);
  memcpy(tmp, in_c, sizeof(cplx) * nh);
  fftplan px, py, pz;
  plan_init(&px, nx); plan_init(&py, ny); plan_init(&pz, nz);
  int mx = nx > ny ? nx : ny; mx = mx > nz ? mx : nz;
  cplx* line = (cplx*)malloc(sizeof(cplx) * mx);
  cplx* work = (cplx*)malloc(sizeof(cplx) * mx);
  for (int y = 0; y < ny; ++y)
    for (int k = 0; k < nxh; ++k) {
      for (int z = 0; z < nz; ++z) line[z] = tmp[((long)z * ny + y) * nxh + k];
      fft1(&pz, line, work, 1);
      for (int z = 0; z < nz; ++z) tmp[((long)z * ny + y) * nxh + k] = line[z];
    }
  for (int z = 0; z < nz; ++z)
    for (int k = 0; k < nxh; ++k) {
      for (int y = 0; y < ny; ++y) line[y] = tmp[((long)z * ny + y) * nxh + k];
      fft1(&py, line, work, 1);
      for (int y = 0; y < ny; ++y) tmp[((long)z * ny + y) * nxh + k] = line[y];
    }
  for (long r = 0; r < (long)ny * nz; ++r) {
    for (int x = 0; x < nx; ++x) {
      int k = x <= nx / 2 ? x : nx - x;
      cplx v = tmp[r * nxh + k];
      if (k == 0 || 2 * k == nx) v.im = 0;
      if (x > nx / 2) v.im = -v.im;
      line[x] = v;
    }
    fft1(&px, line, work, 1);
    for (int x = 0; x < nx; ++x) out[r * nx + x] = line[x].re;
  }
  free(line); free(work); free(tmp);
  plan_free(&px); plan_free(&py); plan_free(&pz);
}

/* complex 1-D FFT of `count` contiguous lines (for unit tests of the FFT itself) */
EXPORT void FN(orc_fft1)(REAL* data_c, int n, int count, int sign) {
  fftplan p;
  plan_init(&p, n);
  cplx* w = (cplx*)malloc(sizeof(cplx) * n);
  for (int i = 0; i < count; ++i) fft1(&p, (cplx*)data_c + (long)i * n, w, sign);
  free(w);
  plan_free(&p);
}

/* Hermitian weight of half-spectrum column kx (full-spectrum multiplicity) */
static inline double herm_w(int kx, int nx) { return (kx == 0 || 2 * kx == nx) ? 1.0 : 2.0; }

/* ------------------------------------------------------------------ CTF */
/* ctfParams constructor (mexFiles/include/core_headers.cuh:63-75) and the plain CTF
 * kernel (mexFiles/utils/ctf.cu:12-66), plus the exposure-filtered variant (:68-130).
 * Arithmetic in REAL. */
typedef struct {
  REAL cs_term, df_term, amp_phase, df1, df2, ast;
} ctfp;

static ctfp ctf_params(REAL wavelength, REAL cs_mm, REAL amp, REAL df1, REAL df2, REAL ast_deg) {
  ctfp p;
  const double PI = 3.14159265358979323;
  p.amp_phase = (REAL)atan((double)amp / sqrt(1.0 - (double)amp * amp));
  p.df1 = (REAL)(0.5 * (df1 + df2));
  p.df2 = (REAL)(0.5 * (df1 - df2));
  p.ast = (REAL)(ast_deg * PI / 180.0 - PI * (double)lrint(ast_deg / 180.0));
  p.cs_term = (REAL)(PI * 0.5 * cs_mm * 1e7 * pow(wavelength, 3));
  p.df_term = (REAL)(PI * wavelength);
  return p;
}

static REAL ctf_value(const ctfp* p, double fx, double fy, int squared) {
  double phi = atan2(fy, fx);
  double r2 = fx * fx + fy * fy;
  double v = sin(p->cs_term * r2 * r2 - p->df_term * r2 * (p->df1 + p->df2 * cos(2.0 * (phi - p->ast))) - p->amp_phase);
  return (REAL)(squared ? v * v : v);
}

/* mexCTF (mexFiles/mexCTF.cu:47-111): out is (half ? nx/2+1 : nx) x ny */
EXPORT void FN(orc_ctf2d)(REAL pix, REAL wavelength, REAL cs_mm, REAL df1, REAL df2, REAL ast_deg, REAL amp,
                          int nx, int ny, int half, int squared, int centred, int use_exposure, REAL radial_weight,
                          REAL exposure, REAL* out) {
  ctfp p = ctf_params(wavelength, cs_mm, amp, df1, df2, ast_deg);
  const int dx = half ? nx / 2 + 1 : nx;
  const int ox = half ? 0 : nx / 2, oy = ny / 2;
  const double fvx = 1.0 / ((double)pix * nx), fvy = 1.0 / ((double)pix * ny);
  for (int y0 = 0; y0 < ny; ++y0)
    for (int x0 = 0; x0 < dx; ++x0) {
      int x = x0, y = y0;
      if (centred) {
        y -= oy;
        if (!half) x -= ox;
      } else {
        if (y > oy) y -= ny;
        if (!half && x > ox) x -= dx;
      }
      double fx = x * fvx, fy = y * fvy;
      double v = ctf_value(&p, fx, fy, squared);
      if (use_exposure) {
        /* ctf.cu:108-127 */
        double rw = radial_weight * (x == 0 ? 0.2 : fabs((double)x));
        double r2 = fx * fx + fy * fy;
        double denom = 0.24499 * pow(r2, -0.8325) + 2.81410;
        v *= rw * exp((-0.5 * exposure) / denom);
      }
      out[(long)y0 * dx + x0] = (REAL)v;
    }
}

/* mexSF3D (mexFiles/mexSF3D.cu:24-78 kernel, :237-276 per-tilt loop): for every tilt the
 * exposure-weighted CTF^2 image (full grid, centred) is sampled bilinearly with a zero
 * border and added to the voxels within 4 px of the tilted central plane with a cosine
 * edge weight.  Exact bilinear weights (the reference's texture uses 8-bit ones). */
EXPORT void FN(orc_sf3d)(int squared, int nx, int ny, int nz, const REAL* pix, const REAL* wl, const REAL* cs,
                         const REAL* df1, const REAL* df2, const REAL* ast, const REAL* ac, int ntilts,
                         const REAL* tilt, const REAL* exposure, const REAL* occupancy, REAL* out) {
  const double PI = 3.14159265358979323;
  memset(out, 0, sizeof(REAL) * (long)nx * ny * nz);
  REAL* img = (REAL*)malloc(sizeof(REAL) * (long)nx * ny);
  const double ssx = (nx % 2 == 0) ? 0.5 : 0.0;
  const double ssy = (ny % 2 == 0) ? 0.5 : 0.0;
  const double ssz = (nz % 2 == 0) ? 0.5 : 0.0;
  for (int t = 0; t < ntilts; ++t) {
    FN(orc_ctf2d)(pix[t], wl[t], cs[t], df1[t], df2[t], ast[t], ac[t], nx, ny, 0, squared, 1, 1, occupancy[t],
                  exposure[t], img);
    const double ang = -(double)tilt[t] * PI / 180.0;
    const double sA = sin(ang), cA = cos(ang);
    for (int y = 0; y < ny; ++y) {
      const double tv = ((double)(y - ny / 2) + ssy) / ny + 0.5; /* normalised (:49) */
      const double ty = tv * ny - 0.5;                            /* texel space */
      for (int x = 0; x < nx; ++x) {
        const double u = (double)x - (double)nx / 2.0;
        const double tw_pre = -u * sA + ssz;
        for (int z = 0; z < nz; ++z) {
          const double w = (double)(z - nz / 2);
          const double tw = tw_pre + w * cA;
          if (tw < -4.0 || tw > 4.0) continue;
          const double zw = (0.5 + 0.5 * cos(tw * (PI / 4.0))) * 0.25;
          double tu = u * cA + w * sA + ssx;
          tu = tu / nx + 0.5;
          const double tx = tu * nx - 0.5;
          /* bilinear, zero border */
          int x0 = (int)floor(tx), y0 = (int)floor(ty);
          double fx = tx - x0, fy = ty - y0, acc = 0;
          for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
              int xi = x0 + dx, yi = y0 + dy;
              if (xi < 0 || yi < 0 || xi >= nx || yi >= ny) continue;
              acc += (dx ? fx : 1 - fx) * (dy ? fy : 1 - fy) * img[(long)yi * nx + xi];
            }
          out[((long)z * ny + y) * nx + x] += (REAL)(zw * acc);
        }
      }
    }
  }
  free(img);
}

/* ------------------------------------------------------------------ particle spectrum */
/* Q = weight .* bandpass .* fftn(particle), Q(0) = 0 (masking/BH_bandLimitCenterNormalize.m:48-55;
 * the reference's final scalar normalisation (:61) cancels in the normalised CC and is
 * not applied).  Returns sum |Q|^2 over the full spectrum. */
EXPORT double FN(orc_particle_spectrum)(const REAL* particle, const REAL* weight, const REAL* bandpass, int n,
                                        REAL* Q_c) {
  const int nh = n / 2 + 1;
  FN(orc_fft3_r2c)(particle, n, n, n, Q_c);
  cplx* Q = (cplx*)Q_c;
  double e = 0;
  for (long i = 0; i < (long)nh * n * n; ++i) {
    double f = 1;
    if (weight) f *= weight[i];
    if (bandpass) f *= bandpass[i];
    if (i == 0) f = 0;
    Q[i].re = (REAL)(Q[i].re * f);
    Q[i].im = (REAL)(Q[i].im * f);
    e += herm_w((int)(i % nh), n) * ((double)Q[i].re * Q[i].re + (double)Q[i].im * Q[i].im);
  }
  return e;
}

/* ------------------------------------------------------------------ normalised translational CC */
/* statistics/BH_multi_xcf_Translational_2.m:35-38 with its four operands, on half spectra (every
 * sum over MATLAB's full spectrum is the Hermitian-weighted sum over the half):
 *   iCCCmap = real(ifftn(refWdg .* rotPART_FT .* REF_FT .* wdgMask))
 *             * numel / sqrt(sum|REF_FT .* wdgMask|^2 * sum|rotPART_FT .* refWdg|^2)
 * where, as at the call site (alignment/BH_alignRaw3d_v2.m:1287-1330):
 *   REF_FT     = conj(R), R = wref .* fftn(mask .* I(M (p - c - t) + c)) with R(0) = 0: the
 *                reference sampled through M with 'forward' semantics and passed through
 *                BH_bandLimitCenterNormalize(.., bandpassFiltREF) (whose final scalar cancels);
 *   rotPART_FT = P, the particle spectrum with P(0) = 0 (BH_bandLimitCenterNormalize output);
 *   wdgMask    = the weight that multiplies the reference spectrum (NULL = 1);
 *   refWdg     = the weight that multiplies the particle spectrum (NULL = 1).
 * The unnormalised inverse transform (no 1/numel) is numel * ifftn.  Writes the map in FFT order
 * (unshifted) and returns 1 / sqrt(E_R E_P). */
static double xcf2_map(const REAL* ref, const REAL* mask, const REAL* wref, int n, const cplx* P,
                       const REAL* ref_wdg, const REAL* wdg_mask, const double M[9], const double shift[3],
                       int interp, REAL* r, cplx* X, REAL* map) {
  const int nh = n / 2 + 1;
  const long nhalf = (long)nh * n * n;
  const int c = n / 2;
  for (int z = 0; z < n; ++z)
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) {
        double s[3];
        sample_pos(M, shift, 1, x, y, z, c, c, c, s);
        REAL v = interp == 1 ? interp_cubic(ref, n, n, n, s[0], s[1], s[2])
                             : interp_linear(ref, n, n, n, s[0], s[1], s[2], interp == 2);
        long i = ((long)z * n + y) * n + x;
        r[i] = mask ? (REAL)(v * mask[i]) : v;
      }
  FN(orc_fft3_r2c)(r, n, n, n, (REAL*)X);
  double ER = 0, EP = 0;
  for (long i = 0; i < nhalf; ++i) {
    const double hw = herm_w((int)(i % nh), n);
    cplx R = X[i];
    if (wref) { R.re *= wref[i]; R.im *= wref[i]; }
    if (i == 0) { R.re = 0; R.im = 0; }
    const cplx ref_ft = {R.re, (REAL)-R.im};                       /* REF_FT = conj(R) */
    const REAL wm = wdg_mask ? wdg_mask[i] : (REAL)1, rw = ref_wdg ? ref_wdg[i] : (REAL)1;
    const cplx rw_ref = {ref_ft.re * wm, ref_ft.im * wm};           /* REF_FT .* wdgMask */
    const cplx p_rw = {P[i].re * rw, P[i].im * rw};                 /* rotPART_FT .* refWdg */
    ER += hw * ((double)rw_ref.re * rw_ref.re + (double)rw_ref.im * rw_ref.im);
    EP += hw * ((double)p_rw.re * p_rw.re + (double)p_rw.im * p_rw.im);
    X[i] = c_mul(p_rw, rw_ref);                                     /* refWdg.*P.*REF_FT.*wdgMask */
  }
  FN(orc_fft3_c2r)((REAL*)X, n, n, n, map);
  return 1.0 / sqrt(ER * EP);
}

/* ------------------------------------------------------------------ orientation search */
/* One CC evaluation per orientation: the normalised map of xcf2_map (BH_multi_xcf_Translational_2.m:
 * 35-38) for M = RotMat (the reference sampled through RotMat', 'forward';
 * BH_alignRaw3d_v2.m:1287-1291) and the masked argmax of BH_multi_xcf_Translational.m:33-42 over
 * shifts s with |s|^2 <= radius^2 (the spherical peakMask); ties go to the smallest fftshifted
 * column-major index (MATLAB max).  Outputs per orientation the CC and the integer shift s
 * (x, y, z).  P: particle half spectrum (complex).  OpenMP over orientations with `nthreads`. */
EXPORT void FN(orc_search)(const REAL* ref, const REAL* mask, const REAL* wref, int n, const REAL* P_c,
                           const REAL* ref_wdg, const REAL* wdg_mask, const double* Mlist, int norient,
                           const double shift[3], int radius, int interp, int nthreads, double* cc_out,
                           int* peak_out) {
  const int nh = n / 2 + 1;
  const long nvox = (long)n * n * n, nhalf = (long)nh * n * n;
  const cplx* P = (const cplx*)P_c;
  const int c = n / 2;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
  {
    REAL* r = (REAL*)malloc(sizeof(REAL) * nvox);
    REAL* map = (REAL*)malloc(sizeof(REAL) * nvox);
    cplx* X = (cplx*)malloc(sizeof(cplx) * nhalf);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
    for (int o = 0; o < norient; ++o) {
      const double norm = xcf2_map(ref, mask, wref, n, P, ref_wdg, wdg_mask, Mlist + 9 * o, shift, interp, r, X, map);
      double best = -INFINITY;
      long best_idx = 0x7fffffffffffL;
      int bs[3] = {0, 0, 0};
      for (int sz = -c; sz < n - c; ++sz)
        for (int sy = -c; sy < n - c; ++sy)
          for (int sx = -c; sx < n - c; ++sx) {
            if (sx * sx + sy * sy + sz * sz > radius * radius) continue;
            long ui = ((long)((sz + n) % n) * n + (sy + n) % n) * n + (sx + n) % n;
            double v = (double)map[ui] * norm;
            long si = ((long)(sz + c) * n + (sy + c)) * n + (sx + c);
            if (v > best || (v == best && si < best_idx)) {
              best = v; best_idx = si;
              bs[0] = sx; bs[1] = sy; bs[2] = sz;
            }
          }
      cc_out[o] = best;
      peak_out[3 * o + 0] = bs[0];
      peak_out[3 * o + 1] = bs[1];
      peak_out[3 * o + 2] = bs[2];
    }
    free(r); free(map); free(X);
  }
}

/* Full normalised CC map (fftshifted, BH_multi_xcf_Translational_2.m:35-38, operands as xcf2_map) for
 * one rotation matrix, followed by the peak-mask / argmax / two-pass centre of mass of
 * BH_multi_xcf_Translational.m:33-97 (peakCOM = 3).  Writes the map (n^3, fftshifted) and the
 * subvoxel peak (x, y, z) relative to the origin; returns the map maximum inside the peak mask. */
EXPORT double FN(orc_xcf_translational)(const REAL* ref, const REAL* mask, const REAL* wref, int n, const REAL* P_c,
                                        const REAL* ref_wdg, const REAL* wdg_mask, const double M[9],
                                        const double shift[3], const REAL* peak_mask, int interp, REAL* map_out,
                                        double peak_out[3]) {
  const int nh = n / 2 + 1;
  const long nvox = (long)n * n * n, nhalf = (long)nh * n * n;
  const int c = n / 2;
  REAL* r = (REAL*)malloc(sizeof(REAL) * nvox);
  REAL* map = (REAL*)malloc(sizeof(REAL) * nvox);
  cplx* X = (cplx*)malloc(sizeof(cplx) * nhalf);
  const double norm = xcf2_map(ref, mask, wref, n, (const cplx*)P_c, ref_wdg, wdg_mask, M, shift, interp, r, X, map);
  /* fftshift into map_out */
  double minv = INFINITY;
  for (int z = 0; z < n; ++z)
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) {
        long ui = ((long)z * n + y) * n + x;
        int zs = (z + c) % n, ys = (y + c) % n, xs = (x + c) % n;
        double v = map[ui] * norm;
        map_out[((long)zs * n + ys) * n + xs] = (REAL)v;
        if (v < minv) minv = v;
      }
  /* peakMask < 0.95 -> min (:33-34); argmax, first index wins */
  long bi = 0;
  double bv = -INFINITY;
  for (long i = 0; i < nvox; ++i) {
    double v = (peak_mask && peak_mask[i] < 0.95) ? minv : (double)map_out[i];
    if (v > bv) { bv = v; bi = i; }
  }
  double pc[3] = {(double)(bi % n), (double)((bi / n) % n), (double)(bi / ((long)n * n))};
  if (bv == bv && bv != 0) {
    for (int it = 0; it < 2; ++it) {
      double base[3];
      for (int d = 0; d < 3; ++d) base[d] = it == 1 ? floor(pc[d] + 0.5) : pc[d];
      double sum = 0, cm[3] = {0, 0, 0};
      for (int dz = -3; dz <= 3; ++dz)
        for (int dy = -3; dy <= 3; ++dy)
          for (int dx = -3; dx <= 3; ++dx) {
            int xi = (int)base[0] + dx, yi = (int)base[1] + dy, zi = (int)base[2] + dz;
            if (xi < 0 || yi < 0 || zi < 0 || xi >= n || yi >= n || zi >= n) continue;
            double v = (peak_mask && peak_mask[((long)zi * n + yi) * n + xi] < 0.95)
                           ? minv : (double)map_out[((long)zi * n + yi) * n + xi];
            v -= minv;
            sum += v; cm[0] += v * dx; cm[1] += v * dy; cm[2] += v * dz;
          }
      for (int d = 0; d < 3; ++d) pc[d] = base[d] + cm[d] / sum;
    }
  }
  for (int d = 0; d < 3; ++d) peak_out[d] = pc[d] - c;
  free(r); free(map); free(X);
  return bv;
}

/* ------------------------------------------------------------------ template search */
/* BH_templateSearch3d_2.m:633-887 for one chunk covering the whole tomogram:
 *   T   = swapQuadrants .* fftn(tomo)(half)                                   (:633-641, :714)
 *   g   = template through defineMatrix([phi,theta,psi-phi],'forward'), shift [1,1,1] (:744)
 *   G   = fftn(g zero-padded to the centre, BH_multi_padVal)                  (:752-756)
 *   cc  = real(ifftn(T .* conj(G)));  cc = cc / std(cc(:))                    (:760-764)
 *   peak(cc > peak) = cc, angle = orientation index (1-based)                 (:851-854)
 * Mlist: 9 doubles per orientation. */
EXPORT void FN(orc_tsearch)(const REAL* tomo, int nx, int ny, int nz, const REAL* tmpl, int t, const double* Mlist,
                            int norient, REAL* peak, REAL* angle) {
  const int nxh = nx / 2 + 1;
  const long nvox = (long)nx * ny * nz, nhalf = (long)nxh * ny * nz;
  cplx* T = (cplx*)malloc(sizeof(cplx) * nhalf);
  cplx* G = (cplx*)malloc(sizeof(cplx) * nhalf);
  REAL* g = (REAL*)malloc(sizeof(REAL) * nvox);
  REAL* rot = (REAL*)malloc(sizeof(REAL) * (long)t * t * t);
  REAL* cc = (REAL*)malloc(sizeof(REAL) * nvox);
  FN(orc_fft3_r2c)(tomo, nx, ny, nz, (REAL*)T);
  /* swapQuadrants: exp(-2 pi i (u (nx/2+1)/nx + v (ny/2+1)/ny + w (nz/2+1)/nz)) on the centred
   * grid u = i - floor(nx/2) of array position i, first nx/2+1 x-positions (:633-641) */
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nxh; ++x) {
        double u = (double)(x - nx / 2) / nx, v = (double)(y - ny / 2) / ny, w = (double)(z - nz / 2) / nz;
        double ph = -2.0 * M_PI * (u * (nx / 2 + 1) + v * (ny / 2 + 1) + w * (nz / 2 + 1));
        cplx e = {(REAL)cos(ph), (REAL)sin(ph)};
        long i = ((long)z * ny + y) * nxh + x;
        T[i] = c_mul(e, T[i]);
      }
  const int pl[3] = {(nx - t) / 2 + ((t % 2) ? (nx - t) % 2 : 0), (ny - t) / 2 + ((t % 2) ? (ny - t) % 2 : 0),
                     (nz - t) / 2 + ((t % 2) ? (nz - t) % 2 : 0)};
  const double sh[3] = {1, 1, 1};
  for (long i = 0; i < nvox; ++i) { peak[i] = -INFINITY; angle[i] = 1; }
  for (int o = 0; o < norient; ++o) {
    FN(orc_rotate)(tmpl, t, t, t, Mlist + 9 * o, 1, sh, 1, 0, rot);
    memset(g, 0, sizeof(REAL) * nvox);
    for (int z = 0; z < t; ++z)
      for (int y = 0; y < t; ++y)
        for (int x = 0; x < t; ++x)
          g[((long)(z + pl[2]) * ny + (y + pl[1])) * nx + (x + pl[0])] = rot[((long)z * t + y) * t + x];
    FN(orc_fft3_r2c)(g, nx, ny, nz, (REAL*)G);
    for (long i = 0; i < nhalf; ++i) {
      cplx a = T[i], b = G[i];
      G[i].re = a.re * b.re + a.im * b.im;
      G[i].im = a.im * b.re - a.re * b.im;
    }
    FN(orc_fft3_c2r)((REAL*)G, nx, ny, nz, cc);
    double s = 0, s2 = 0;
    for (long i = 0; i < nvox; ++i) s += cc[i];
    const double mean = s / nvox;
    for (long i = 0; i < nvox; ++i) s2 += ((double)cc[i] - mean) * ((double)cc[i] - mean);
    const double sd = sqrt(s2 / (nvox - 1));
    for (long i = 0; i < nvox; ++i) {
      REAL v = (REAL)(cc[i] / sd);
      if (peak[i] < v) { peak[i] = v; angle[i] = (REAL)(o + 1); }
    }
  }
  free(T); free(G); free(g); free(rot); free(cc);
}

/* ------------------------------------------------------------------ pose CC and gradient */
/* Zero-lag normalised CC of the rotated, shifted reference (tricubic, 'forward' sampling)
 * against the real-space particle template h = C2R(Q) and its exact gradient w.r.t. the
 * 9 matrix entries and the 3 shift components.  E_R is the DC-free energy
 * n^3 sum r^2 - (sum r)^2 (Parseval).  Returns CC; dM (9, column-major) and dt (3). */
EXPORT double FN(orc_cc_pose_interp)(const REAL* ref, const REAL* mask, int n, const REAL* h, double EP,
                                     const double M[9], const double t[3], int interp, double dM[9], double dt[3]);

EXPORT double FN(orc_cc_pose)(const REAL* ref, const REAL* mask, int n, const REAL* h, double EP, const double M[9],
                              const double t[3], double dM[9], double dt[3]) {
  return FN(orc_cc_pose_interp)(ref, mask, n, h, EP, M, t, 1, dM, dt);
}

/* As orc_cc_pose with interp 0 = trilinear (interpn) or 1 = tricubic. */
EXPORT double FN(orc_cc_pose_interp)(const REAL* ref, const REAL* mask, int n, const REAL* h, double EP,
                                     const double M[9], const double t[3], int interp, double dM[9], double dt[3]) {
  const int c = n / 2;
  const long nvox = (long)n * n * n;
  double* r = (double*)malloc(sizeof(double) * nvox);
  double* gs = (double*)malloc(sizeof(double) * nvox * 3);
  double A = 0, S1 = 0, S2 = 0;
  for (int z = 0; z < n; ++z)
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) {
        double s[3], g[3];
        sample_pos(M, t, 1, x, y, z, c, c, c, s);
        long i = ((long)z * n + y) * n + x;
        double v = interp == 1 ? interp_cubic_grad(ref, n, n, n, s[0], s[1], s[2], g)
                               : interp_linear_grad(ref, n, n, n, s[0], s[1], s[2], g);
        double m = mask ? (double)mask[i] : 1.0;
        r[i] = m * v;
        gs[3 * i] = m * g[0]; gs[3 * i + 1] = m * g[1]; gs[3 * i + 2] = m * g[2];
        A += r[i] * (double)h[i];
        S1 += r[i];
        S2 += r[i] * r[i];
      }
  const double N3 = (double)nvox;
  const double ER = N3 * S2 - S1 * S1;
  const double cc = A / sqrt(ER * EP);
  for (int k = 0; k < 9; ++k) dM[k] = 0;
  dt[0] = dt[1] = dt[2] = 0;
  for (int z = 0; z < n; ++z)
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) {
        long i = ((long)z * n + y) * n + x;
        /* dCC/dr(p) */
        double gr = (double)h[i] / sqrt(ER * EP) - cc / ER * (N3 * r[i] - S1);
        double u[3] = {(double)(x - c) - t[0], (double)(y - c) - t[1], (double)(z - c) - t[2]};
        /* s = M u + c  -> ds_i/dM_ij = u_j ; ds/dt = -M */
        for (int a = 0; a < 3; ++a) {
          double ga = gr * gs[3 * i + a];
          for (int b = 0; b < 3; ++b) dM[a + 3 * b] += ga * u[b];
          for (int b = 0; b < 3; ++b) dt[b] -= ga * M[a + 3 * b];
        }
      }
  free(r); free(gs);
  return cc;
}
