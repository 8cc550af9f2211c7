// tsearch.cu -- template matching over a whole tomogram (BH_templateSearch3d_2.m:633-887).
//
// Once per tomogram: T = swapQuadrants .* fftn(tomo) (half spectrum, :633-641, :714).
// Per orientation o (1-based index, :851-854):
//   g   = template sampled through defineMatrix([phi,theta,psi-phi],'forward') with shift [1,1,1]
//         ('forward' semantics, :744), placed in the centre of the volume (BH_multi_padVal, :752)
//   X   = T .* conj(fftn(g))
//   cc  = real(ifftn(X)) / std(cc)     std from the spectrum by Parseval, accumulated in FP64
//   peak(peak < cc) = cc, angle = o
// The template volume is never materialised at full size.  Per orientation:
//   k_ts_rows    samples the rotated template straight into the x transforms of its t x t rows
//                (two rows per complex FFT), written into a t-plane buffer whose other rows stay 0;
//   k_cols (y)   the y transforms of those t planes;
//   k_ts_zfused  per tile of (ky, kx) z-lines: forward z transform of the t non-zero planes
//                (the rest are zeros), X = T .* conj(G) with the FP64 map statistics, inverse z;
//   k_cols (y)   inverse y;  k_ts_c2r_mip: C2R along x fused with the std normalisation and the
//                MIP update.
// Per orientation this reads the tomogram spectrum once and moves the full-size spectrum through
// HBM four times (z out, y in / out, x in) instead of the seven passes of an unfused pipeline.
#include <math.h>

#include <algorithm>
#include <new>
#include <vector>

#include "fft_passes.cuh"
#include "interp.cuh"

namespace emc {

struct TsGeom {
  int nx, ny, nz, nxh;
  int t;            // template edge
  int pl[3];        // template offset inside the volume (BH_multi_padVal low pad)
  float m[9];       // sampling matrix rows
};

// Rotated template sampled into the x transforms of its rows: pair p of the t * ceil(t/2) row
// pairs is rows (2q, 2q+1) of template plane zl; the line z[n] = a[n] + i b[n] holds the template
// at x = n - pl[0] (zero outside), and the two half spectra go to rows pl[1] + 2q (+1) of plane zl
// of ht ([t][ny][nxh]).  Sampling: 'forward' with shift [1,1,1], u = p - c - 1
// (BH_templateSearch3d_2.m:744), interpn-style trilinear.
template <int L, int P>
__global__ void __launch_bounds__(256) k_ts_rows(const float* __restrict__ tmpl, const TsGeom g,
                                                 float2* __restrict__ ht, const float2* __restrict__ g_tw) {
  constexpr int TEAMS = rows_teams(L, P);
  constexpr int PAD = line_pad(L);
  __shared__ float2 s_tw[L];
  __shared__ float2 s_line[TEAMS][row_line_len(L)];
  load_twiddles<L>(s_tw, g_tw);
  __syncthreads();
  const int team = threadIdx.x / P, lane = threadIdx.x % P;
  const int hp = (g.t + 1) / 2;
  const long npairs = (long)g.t * hp;
  const int c = g.t / 2;
  for (long pair0 = (long)blockIdx.x * TEAMS; pair0 < npairs; pair0 += (long)gridDim.x * TEAMS) {
    const long pair = pair0 + team;
    const bool active = pair < npairs;
    const int zl = active ? (int)(pair / hp) : 0, q = active ? (int)(pair % hp) : 0;
    const int ya = 2 * q, yb = 2 * q + 1;
    const bool has_b = yb < g.t;
    float2* buf = s_line[team];
    if (active) {
      const float w2 = (float)(zl - c) - 1.f;
      const float wa = (float)(ya - c) - 1.f, wb = (float)(yb - c) - 1.f;
      for (int n = lane; n < L; n += P) {
        const int px = n - g.pl[0];
        float va = 0.f, vb = 0.f;
        if (px >= 0 && px < g.t) {
          const float u = (float)(px - c) - 1.f;
          {
            const float sx = fmaf(g.m[0], u, fmaf(g.m[1], wa, g.m[2] * w2)) + (float)c;
            const float sy = fmaf(g.m[3], u, fmaf(g.m[4], wa, g.m[5] * w2)) + (float)c;
            const float sz = fmaf(g.m[6], u, fmaf(g.m[7], wa, g.m[8] * w2)) + (float)c;
            va = sample_linear(tmpl, g.t, g.t, g.t, sx, sy, sz);
          }
          if (has_b) {
            const float sx = fmaf(g.m[0], u, fmaf(g.m[1], wb, g.m[2] * w2)) + (float)c;
            const float sy = fmaf(g.m[3], u, fmaf(g.m[4], wb, g.m[5] * w2)) + (float)c;
            const float sz = fmaf(g.m[6], u, fmaf(g.m[7], wb, g.m[8] * w2)) + (float)c;
            vb = sample_linear(tmpl, g.t, g.t, g.t, sx, sy, sz);
          }
        }
        buf[lpos<PAD>(n)] = make_float2(va, vb);
      }
    }
    __syncwarp();
    fft_line<L, -1, P, PAD>(buf, 1, lane, s_tw, active);
    if (active) {
      float2* oa = ht + ((size_t)zl * g.ny + g.pl[1] + ya) * g.nxh;
      float2* ob = oa + g.nxh;
      for (int k = lane; k <= L / 2; k += P) {
        const float2 zk = buf[lpos<PAD>(k)], zm = buf[lpos<PAD>((L - k) % L)];
        oa[k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        if (has_b) ob[k] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
      }
    }
    __syncwarp();
  }
}

// Per tile of TT consecutive (ky, kx) z-lines: G = FFT_z of the t planes at z = pl[2].. (zeros
// elsewhere), X = T .* conj(G), inverse FFT_z into s.  stats[0] += sum over the full spectrum of
// |X|^2 (Hermitian weights), stats[1] = X(0).  The product and statistics are formed in registers
// between the two transforms (fft_line_fwd_mul_inv).
// Resident CTAs per SM asked of the compiler: 20 warps' worth when a lane holds at most 16 complex
// values per stage (the register cap then leaves room for them), else no constraint.
constexpr int zfused_min_blocks(int L, int P, int TT) {
  return stage_values(L, P) <= 16 && 640 / (P * TT) > 1 ? 640 / (P * TT) : 1;
}

template <int L, int P, int TT>
__global__ void __launch_bounds__(P * TT, zfused_min_blocks(L, P, TT)) k_ts_zfused(const float2* __restrict__ gt, const float2* __restrict__ T,
                                                      float2* __restrict__ s, const TsGeom g,
                                                      double* __restrict__ stats, const float2* __restrict__ g_tw) {
  extern __shared__ float2 smem[];
  constexpr int TP = TT + 1;
  constexpr int PAD = line_pad(L);
  float2* s_tw = smem;
  float2* tile = smem + L;                                // [padded L][TP], element n of line t at lpos<PAD>(n) * TP + t
  float2* s_t = tile + (size_t)padded_len(L, PAD) * TP;  // [L][TT], the tomogram spectrum of the tile's lines
  static_assert((P * TT) % 32 == 0, "the statistics reduction needs whole warps");
  __shared__ double red[32];
  load_twiddles<L>(s_tw, g_tw);
  const long inner = (long)g.ny * g.nxh, stride = inner;
  const long i0 = (long)blockIdx.x * TT;
  constexpr int NT = P * TT;
  constexpr int IT = (L * TT + NT - 1) / NT;
  // the tomogram spectrum of this tile, copied asynchronously while the template planes load
#pragma unroll
  for (int k = 0; k < IT; ++k) {
    const int idx = threadIdx.x + k * NT;
    const int n = idx / TT, t = idx % TT;
    if (idx < L * TT && i0 + t < inner) cp_async8(s_t + idx, T + (long)n * stride + i0 + t);
  }
  cp_async_commit();
  {
    float2 v[IT];
#pragma unroll
    for (int k = 0; k < IT; ++k) {
      const int idx = threadIdx.x + k * NT;
      const int n = idx / TT, t = idx % TT;
      const long i = i0 + t;
      v[k] = make_float2(0.f, 0.f);
      if (idx < L * TT && i < inner && n >= g.pl[2] && n < g.pl[2] + g.t) v[k] = gt[(long)(n - g.pl[2]) * stride + i];
    }
#pragma unroll
    for (int k = 0; k < IT; ++k) {
      const int idx = threadIdx.x + k * NT;
      if (idx < L * TT) tile[lpos<PAD>(idx / TT) * TP + idx % TT] = v[k];
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  const int team = threadIdx.x / P, lane = threadIdx.x % P;
  const long i = i0 + team;
  const bool line_active = i < inner;
  const double hw = ((int)(i % g.nxh) == 0 || 2 * (int)(i % g.nxh) == g.nx) ? 1.0 : 2.0;
  // forward z transform of the template planes, X = T .* conj(G) and its statistics in registers,
  // inverse z transform (fft_line_fwd_mul_inv).  Each lane sums its elements' |X|^2 in FP32 (L / P
  // of them), the lanes' sums are accumulated in FP64.
  float ef = 0.f;
  fft_line_fwd_mul_inv<L, P, PAD>(tile + team, TP, lane, s_tw, line_active, [&](int n, float2 gz) {
    const float2 x = cmulc(s_t[n * TT + team], gz);
    ef = fmaf(x.x, x.x, fmaf(x.y, x.y, ef));
    if (i == 0 && n == 0) stats[1] = (double)x.x;
    return x;
  });
  double e = hw * (double)ef;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < NT / 32; ++w) tot += red[w];
    atomicAdd(stats, tot);
  }
  for (int idx = threadIdx.x; idx < L * TT; idx += NT) {
    const int n = idx / TT, t = idx % TT;
    if (i0 + t < inner) s[(long)n * stride + i0 + t] = tile[lpos<PAD>(n) * TP + t];
  }
}

// Last inverse pass (C2R along x) fused with the std normalisation and the MIP update.  Each team
// (one warp at L = 512) walks its row pairs with the next pair's two spectrum rows copied into a
// second shared buffer (cp.async) while the current pair is transformed, and issues the current
// maxima's loads before its transform, so neither load waits in front of the arithmetic.
template <int L, int P>
struct C2rMipSmem {
  static constexpr int TEAMS = rows_teams(L, P);
  static constexpr int LH = L / 2 + 1;
  static constexpr size_t bytes =
      sizeof(float2) * ((size_t)L + (size_t)TEAMS * row_line_len(L) + 2 * (size_t)TEAMS * 2 * LH);
};

template <int L, int P>
__global__ void __launch_bounds__(256) k_ts_c2r_mip(const float2* __restrict__ in, long nrows,
                                                    const double* __restrict__ stats, long nvox, float angle_id,
                                                    float* __restrict__ peak, float* __restrict__ angle,
                                                    const float2* __restrict__ g_tw) {
  constexpr int TEAMS = rows_teams(L, P);
  constexpr int PAD = line_pad(L);
  constexpr int LH = L / 2 + 1;
  constexpr int RLL = row_line_len(L);
  extern __shared__ float2 c2r_smem[];
  float2* s_tw = c2r_smem;
  float2* s_lines = s_tw + L;                  // [TEAMS][RLL]
  float2* s_spec = s_lines + TEAMS * RLL;      // [2][TEAMS][2 * LH]: rows a, b of a pair
  load_twiddles<L>(s_tw, g_tw);
  // map statistics from the spectrum: mean = X(0), sum m^2 = nvox * sum_full |X|^2
  const double mean = stats[1];
  const double var = (stats[0] * (double)nvox - (double)nvox * mean * mean) / (double)(nvox - 1);
  const float inv_sd = var > 0.0 ? (float)(1.0 / sqrt(var)) : 0.f;
  __syncthreads();
  const int team = threadIdx.x / P, lane = threadIdx.x % P;
  const long npairs = (nrows + 1) / 2;
  const long stride = (long)gridDim.x * TEAMS;
  float2* buf = s_lines + team * RLL;
  // rows 2 pair, 2 pair + 1 of the spectrum into sb (one commit group per call, possibly empty)
  auto prefetch = [&](long pair, float2* sb) {
    if (pair < npairs) {
      const long ra = 2 * pair, rb = 2 * pair + 1;
      for (int k = lane; k < LH; k += P) {
        cp_async8(sb + k, in + ra * LH + k);
        if (rb < nrows) cp_async8(sb + LH + k, in + rb * LH + k);
      }
    }
    cp_async_commit();
  };
  int cur = 0;
  prefetch((long)blockIdx.x * TEAMS + team, s_spec + (size_t)team * 2 * LH);
  for (long pair0 = (long)blockIdx.x * TEAMS; pair0 < npairs; pair0 += stride) {
    const long pair = pair0 + team;
    const bool active = pair < npairs;
    const long ra = 2 * pair, rb = 2 * pair + 1;
    const bool has_b = rb < nrows;
    prefetch(pair + stride, s_spec + ((size_t)(cur ^ 1) * TEAMS + team) * 2 * LH);
    // the current maxima of both rows, in flight during the transform
    constexpr int NE = (L + P - 1) / P;
    float pa[NE], pb[NE];
#pragma unroll
    for (int k = 0; k < NE; ++k) {
      const int n = lane + k * P;
      pa[k] = (active && n < L) ? peak[ra * L + n] : 0.f;
      pb[k] = (active && has_b && n < L) ? peak[rb * L + n] : 0.f;
    }
    cp_async_wait<1>();  // this pair's rows (the next pair's may still be in flight)
    __syncwarp();
    const float2* a = s_spec + ((size_t)cur * TEAMS + team) * 2 * LH;
    const float2* b = a + LH;
    // Hermitian extension of rows a and b packed as a + i b
    fft_line_in<L, 1, P, PAD>(
        [&](int n) {
          const bool lower = n <= L / 2;
          const int k = lower ? n : L - n;
          float2 A = a[k];
          float2 B = has_b ? b[k] : make_float2(0.f, 0.f);
          if (k == 0 || 2 * k == L) { A.y = 0.f; B.y = 0.f; }
          if (!lower) { A.y = -A.y; B.y = -B.y; }
          return make_float2(A.x - B.y, A.y + B.x);
        },
        buf, 1, lane, s_tw, active);
    if (active) {
#pragma unroll
      for (int k = 0; k < NE; ++k) {
        const int n = lane + k * P;
        if (n >= L) break;
        const float2 z = buf[lpos<PAD>(n)];
        const float va = z.x * inv_sd;
        if (pa[k] < va) { peak[ra * L + n] = va; angle[ra * L + n] = angle_id; }
        if (has_b) {
          const float vb = z.y * inv_sd;
          if (pb[k] < vb) { peak[rb * L + n] = vb; angle[rb * L + n] = angle_id; }
        }
      }
    }
    __syncwarp();  // this pair's spectrum rows have been read; the next prefetch reuses the buffer
    cur ^= 1;
  }
  cp_async_wait<0>();
}

__global__ void k_ts_init(float* __restrict__ peak, float* __restrict__ angle, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    peak[i] = -INFINITY;
    angle[i] = 1.f;
  }
}

__global__ void k_ts_ramp(float2* __restrict__ T, const float2* __restrict__ ex, const float2* __restrict__ ey,
                          const float2* __restrict__ ez, int nxh, int ny, int nz) {
  const long total = (long)nz * ny * nxh;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nxh), y = (int)((i / nxh) % ny), z = (int)(i / ((long)nxh * ny));
    T[i] = cmul(cmul(ex[x], ey[y]), cmul(ez[z], T[i]));
  }
}

template <int L>
static emc_status launch_c2r_mip(const float2* in, long nrows, const double* stats, long nvox, float angle_id,
                                 float* peak, float* angle, cudaStream_t st) {
  constexpr int P = team_size(L);
  constexpr int TEAMS = rows_teams(L, P);
  const float2* tw = device_twiddles(L);
  if (!tw) return EMC_E_CUDA;
  const long npairs = (nrows + 1) / 2;
  constexpr size_t smem = C2rMipSmem<L, P>::bytes;
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64) return EMC_E_CUDA;
  if (smem > 48 * 1024 && !attr_set[dev]) {
    EMC_CUDA(cudaFuncSetAttribute(k_ts_c2r_mip<L, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set[dev] = true;
  }
  const int grid = (int)std::max(1L, std::min((npairs + TEAMS - 1) / TEAMS, 8L * device_sm_count()));
  k_ts_c2r_mip<L, P><<<grid, TEAMS * P, smem, st>>>(in, nrows, stats, nvox, angle_id, peak, angle, tw);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

static emc_status c2r_mip_any(int L, const float2* in, long nrows, const double* stats, long nvox, float angle_id,
                              float* peak, float* angle, cudaStream_t st) {
  switch (L) {
#define X(n) case n: return launch_c2r_mip<n>(in, nrows, stats, nvox, angle_id, peak, angle, st);
    EMC_FOR_EACH_LENGTH(X)
#undef X
  }
  set_error("template search: edge %d not supported", L);
  return EMC_E_UNSUPPORTED;
}

template <int L>
static emc_status launch_ts_rows(const float* tmpl, const TsGeom& g, float2* ht, cudaStream_t st) {
  constexpr int P = team_size(L);
  constexpr int TEAMS = rows_teams(L, P);
  const float2* tw = device_twiddles(L);
  if (!tw) return EMC_E_CUDA;
  const long npairs = (long)g.t * ((g.t + 1) / 2);
  const int grid = (int)std::max(1L, std::min((npairs + TEAMS - 1) / TEAMS, 8L * device_sm_count()));
  k_ts_rows<L, P><<<grid, TEAMS * P, 0, st>>>(tmpl, g, ht, tw);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

static emc_status ts_rows_any(int L, const float* tmpl, const TsGeom& g, float2* ht, cudaStream_t st) {
  switch (L) {
#define X(n) case n: return launch_ts_rows<n>(tmpl, g, ht, st);
    EMC_FOR_EACH_LENGTH(X)
#undef X
  }
  set_error("template search: edge %d not supported", L);
  return EMC_E_UNSUPPORTED;
}

template <int L>
static emc_status launch_ts_zfused(const float2* gt, const float2* T, float2* s, const TsGeom& g, double* stats,
                                   cudaStream_t st) {
  using C = ColsCfg<L>;
  const float2* tw = device_twiddles(L);
  if (!tw) return EMC_E_CUDA;
  // Narrow tiles (8 lines, or one warp when the team is smaller than 4 lanes) keep several CTAs
  // resident per SM, so one CTA's loads overlap another's transforms.
  constexpr int TT = C::P >= 4 ? 8 : 32 / C::P;
  auto kern = k_ts_zfused<L, C::P, TT>;
  constexpr size_t smem = sizeof(float2) * (L + (size_t)padded_len(L, line_pad(L)) * (TT + 1) + (size_t)L * TT);
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64) return EMC_E_CUDA;
  if (smem > 48 * 1024 && !attr_set[dev]) {
    EMC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set[dev] = true;
  }
  const long inner = (long)g.ny * g.nxh;
  kern<<<(unsigned)((inner + TT - 1) / TT), C::P * TT, smem, st>>>(gt, T, s, g, stats, tw);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

static emc_status ts_zfused_any(int L, const float2* gt, const float2* T, float2* s, const TsGeom& g, double* stats,
                                cudaStream_t st) {
  switch (L) {
#define X(n) case n: return launch_ts_zfused<n>(gt, T, s, g, stats, st);
    EMC_FOR_EACH_LENGTH(X)
#undef X
  }
  set_error("template search: edge %d not supported", L);
  return EMC_E_UNSUPPORTED;
}

}  // namespace emc

struct emc_tsearch_s {
  int nx, ny, nz;
  float2* T = nullptr;      // tomogram spectrum with the phase ramp
  float2* G = nullptr;      // template spectrum / product
  float2* S = nullptr;      // C2R scratch
  float2* ht = nullptr;     // x transforms of the template rows: [t][ny][nxh], other rows 0
  int ht_t = 0;
  double* stats = nullptr;  // per orientation: sum |X|^2, X(0)
};

extern "C" {

emc_status emc_tsearch_create(const float* d_tomo, int nx, int ny, int nz, emc_tsearch_t* out, void* stream) {
  EMC_CHECK_ARG(d_tomo && out, "emc_tsearch_create: null argument");
  *out = nullptr;
  EMC_CHECK_ARG(emc::fft_length_supported(nx) && emc::fft_length_supported(ny) && emc::fft_length_supported(nz) &&
                    nx >= 2 && ny >= 2 && nz >= 2,
                "emc_tsearch_create: dims %d %d %d must be 2^a 3^b in [2, 512]", nx, ny, nz);
  cudaStream_t st = emc::as_stream(stream);
  emc_tsearch_s* h = new (std::nothrow) emc_tsearch_s();
  EMC_CHECK_ARG(h, "emc_tsearch_create: host allocation failed");
  h->nx = nx; h->ny = ny; h->nz = nz;
  const size_t nh = (size_t)(nx / 2 + 1) * ny * nz;
  if (cudaMalloc(&h->T, nh * sizeof(float2)) || cudaMalloc(&h->G, nh * sizeof(float2)) ||
      cudaMalloc(&h->S, nh * sizeof(float2)) || cudaMalloc(&h->stats, 2 * sizeof(double))) {
    emc_tsearch_destroy(h);
    emc::set_error("emc_tsearch_create: device allocation failed");
    return EMC_E_OOM;
  }
  emc_status rs = emc::fft3_r2c(d_tomo, h->T, nx, ny, nz, 1, st);
  if (rs != EMC_OK) {
    emc_tsearch_destroy(h);
    return rs;
  }
  // swapQuadrants: exp(-2 pi i sum_a (i_a - floor(n_a/2)) (floor(n_a/2)+1) / n_a) per axis (FP64)
  auto axis = [](int n, int len) {
    std::vector<float2> v(len);
    for (int i = 0; i < len; ++i) {
      const double ph = -2.0 * M_PI * (double)(i - n / 2) * (double)(n / 2 + 1) / (double)n;
      v[i] = make_float2((float)cos(ph), (float)sin(ph));
    }
    return v;
  };
  std::vector<float2> ex = axis(nx, nx / 2 + 1), ey = axis(ny, ny), ez = axis(nz, nz);
  float2* d_tab = nullptr;
  const size_t nt = ex.size() + ey.size() + ez.size();
  EMC_CUDA(cudaMallocAsync(&d_tab, nt * sizeof(float2), st));
  EMC_CUDA(cudaMemcpyAsync(d_tab, ex.data(), ex.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
  EMC_CUDA(cudaMemcpyAsync(d_tab + ex.size(), ey.data(), ey.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
  EMC_CUDA(cudaMemcpyAsync(d_tab + ex.size() + ey.size(), ez.data(), ez.size() * sizeof(float2),
                           cudaMemcpyHostToDevice, st));
  emc::k_ts_ramp<<<4 * emc::device_sm_count(), 256, 0, st>>>(h->T, d_tab, d_tab + ex.size(),
                                                             d_tab + ex.size() + ey.size(), nx / 2 + 1, ny, nz);
  EMC_LAUNCH_CHECK();
  EMC_CUDA(cudaStreamSynchronize(st));  // host tables must outlive the copies
  cudaFreeAsync(d_tab, st);
  *out = h;
  return EMC_OK;
}

emc_status emc_tsearch_run(emc_tsearch_t h, const float* d_template, int t, const double* ptp, int n_orient,
                           float* d_peak, float* d_angle, void* stream) {
  EMC_CHECK_ARG(h && d_template && ptp && d_peak && d_angle, "emc_tsearch_run: null argument");
  EMC_CHECK_ARG(t >= 1 && t <= h->nx && t <= h->ny && t <= h->nz, "emc_tsearch_run: template %d too large", t);
  EMC_CHECK_ARG(n_orient >= 1, "emc_tsearch_run: no orientations");
  cudaStream_t st = emc::as_stream(stream);
  const int nx = h->nx, ny = h->ny, nz = h->nz, nxh = nx / 2 + 1;
  const long nvox = (long)nx * ny * nz;
  if (h->ht_t != t) {
    if (h->ht) cudaFree(h->ht);
    h->ht = nullptr;
    h->ht_t = 0;
    const size_t bytes = sizeof(float2) * (size_t)t * ny * nxh;
    EMC_CUDA(cudaMalloc(&h->ht, bytes));
    EMC_CUDA(cudaMemsetAsync(h->ht, 0, bytes, st));  // rows outside the template stay zero
    h->ht_t = t;
  }
  emc::TsGeom g;
  g.nx = nx; g.ny = ny; g.nz = nz; g.nxh = nxh; g.t = t;
  // BH_multi_padVal(t, n): low pad floor((n-t)/2) + (t odd) * ((n-t) odd)
  const int dims[3] = {nx, ny, nz};
  for (int a = 0; a < 3; ++a) g.pl[a] = (dims[a] - t) / 2 + ((t % 2) ? (dims[a] - t) % 2 : 0);
  const int blocks = 4 * emc::device_sm_count();
  emc::k_ts_init<<<blocks, 256, 0, st>>>(d_peak, d_angle, nvox);
  EMC_LAUNCH_CHECK();
  for (int o = 0; o < n_orient; ++o) {
    const double ang[3] = {ptp[3 * o], ptp[3 * o + 1], ptp[3 * o + 2] - ptp[3 * o]};
    double M[9];
    EMC_TRY(emc_define_matrix(ang, 0, M));
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) g.m[3 * i + j] = (float)M[i + 3 * j];
    // 1. rotated template sampled into the x transforms of its rows, 2. y transforms of its planes
    EMC_TRY(emc::ts_rows_any(nx, d_template, g, h->ht, st));
    EMC_TRY(emc::launch_cols(ny, -1, h->ht, h->G, nxh, nxh, t, (long)ny * nxh, st));
    // 3. z transform of the t planes, X = T conj(G) and its statistics, inverse z
    EMC_CUDA(cudaMemsetAsync(h->stats, 0, 2 * sizeof(double), st));
    EMC_TRY(emc::ts_zfused_any(nz, h->G, h->T, h->S, g, h->stats, st));
    // 4. inverse y, then C2R along x fused with std normalisation and the MIP update
    EMC_TRY(emc::launch_cols(ny, 1, h->S, h->S, nxh, nxh, nz, (long)ny * nxh, st));
    EMC_TRY(emc::c2r_mip_any(nx, h->S, (long)ny * nz, h->stats, nvox, (float)(o + 1), d_peak, d_angle, st));
  }
  return EMC_OK;
}

emc_status emc_tsearch_destroy(emc_tsearch_t h) {
  if (!h) return EMC_OK;
  cudaFree(h->T);
  cudaFree(h->G);
  cudaFree(h->S);
  cudaFree(h->ht);
  cudaFree(h->stats);
  delete h;
  return EMC_OK;
}

}  // extern "C"
