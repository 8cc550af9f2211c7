// tsearch.cu -- template matching over a whole tomogram (BH_templateSearch3d_2.m:633-887).
//
// Once per tomogram: T = swapQuadrants .* fftn(tomo) (half spectrum, :633-641, :714).
// Per orientation o (1-based index, :851-854):
//   g   = template sampled through defineMatrix([phi,theta,psi-phi],'forward') with shift [1,1,1]
//         ('forward' semantics, :744), placed in the centre of the volume (BH_multi_padVal, :752)
//   X   = T .* conj(fftn(g))
//   cc  = real(ifftn(X)) / std(cc)     std from the spectrum by Parseval, accumulated in FP64
//   peak(peak < cc) = cc, angle = o
// The template volume is never materialised at full size: its spectrum is built with a pruned
// forward transform (rows and planes that are identically zero are skipped), and the MIP update
// is fused into the last inverse pass.
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

// Rotated template written into the rows it occupies of a real buffer laid out as
// [t (z) planes][ny][nx] for the z planes pl[2]..pl[2]+t-1 only (rows outside the template's
// y/x footprint are zero).
__global__ void k_ts_place(const float* __restrict__ tmpl, const TsGeom g, float* __restrict__ slab) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int zl = blockIdx.z;
  if (x >= g.nx) return;
  float v = 0.f;
  const int px = x - g.pl[0], py = y - g.pl[1];
  if (px >= 0 && px < g.t && py >= 0 && py < g.t) {
    const int c = g.t / 2;
    // 'forward' with shift [1,1,1]: u = p - c - 1
    const float u = (float)(px - c) - 1.f, w1 = (float)(py - c) - 1.f, w2 = (float)(zl - c) - 1.f;
    const float sx = fmaf(g.m[0], u, fmaf(g.m[1], w1, g.m[2] * w2)) + (float)c;
    const float sy = fmaf(g.m[3], u, fmaf(g.m[4], w1, g.m[5] * w2)) + (float)c;
    const float sz = fmaf(g.m[6], u, fmaf(g.m[7], w1, g.m[8] * w2)) + (float)c;
    v = sample_linear(tmpl, g.t, g.t, g.t, sx, sy, sz);
  }
  slab[((long)zl * g.ny + y) * g.nx + x] = v;
}

// Expand the t forward-transformed planes (z = pl[2] .. pl[2]+t-1) into the full z extent with
// zeros elsewhere, so that the z pass can run in place.
__global__ void k_ts_zero_planes(float2* __restrict__ G, const TsGeom g) {
  const long plane = (long)g.ny * g.nxh;
  const long total = plane * g.nz;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int z = (int)(i / plane);
    if (z < g.pl[2] || z >= g.pl[2] + g.t) G[i] = make_float2(0.f, 0.f);
  }
}

// X = T .* conj(G) in place in G; FP64 sums for the map statistics: sum_full |X|^2 and X(0).
__global__ void k_ts_multiply(const float2* __restrict__ T, float2* __restrict__ G, const TsGeom g,
                              double* __restrict__ stats) {
  __shared__ double red[32];
  const long total = (long)g.nz * g.ny * g.nxh;
  double e = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const float2 x = cmulc(T[i], G[i]);
    G[i] = x;
    const int kx = (int)(i % g.nxh);
    e += (kx == 0 || 2 * kx == g.nx ? 1.0 : 2.0) * ((double)x.x * x.x + (double)x.y * x.y);
    if (i == 0) stats[1] = (double)x.x;
  }
  double v = e;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    atomicAdd(stats, t);
  }
}

// Last inverse pass (C2R along x) fused with the std normalisation and the MIP update.
template <int L, int P>
__global__ void __launch_bounds__(256) k_ts_c2r_mip(const float2* __restrict__ in, long nrows,
                                                    const double* __restrict__ stats, long nvox, float angle_id,
                                                    float* __restrict__ peak, float* __restrict__ angle,
                                                    const float2* __restrict__ g_tw) {
  constexpr int TEAMS = rows_teams(L, P);
  constexpr int LH = L / 2 + 1;
  __shared__ float2 s_tw[L];
  __shared__ float2 s_line[TEAMS][L + 1];
  load_twiddles<L>(s_tw, g_tw);
  // map statistics from the spectrum: mean = X(0), sum m^2 = nvox * sum_full |X|^2
  const double mean = stats[1];
  const double var = (stats[0] * (double)nvox - (double)nvox * mean * mean) / (double)(nvox - 1);
  const float inv_sd = var > 0.0 ? (float)(1.0 / sqrt(var)) : 0.f;
  __syncthreads();
  const int team = threadIdx.x / P, lane = threadIdx.x % P;
  const long npairs = (nrows + 1) / 2;
  for (long pair0 = (long)blockIdx.x * TEAMS; pair0 < npairs; pair0 += (long)gridDim.x * TEAMS) {
    const long pair = pair0 + team;
    const bool active = pair < npairs;
    const long ra = 2 * pair, rb = 2 * pair + 1;
    const bool has_b = rb < nrows;
    float2* buf = s_line[team];
    if (active) {
      const float2* a = in + ra * LH;
      const float2* b = in + rb * LH;
      for (int n = lane; n < L; n += P) {
        const bool lower = n <= L / 2;
        const int k = lower ? n : L - n;
        float2 A = a[k];
        float2 B = has_b ? b[k] : make_float2(0.f, 0.f);
        if (k == 0 || 2 * k == L) { A.y = 0.f; B.y = 0.f; }
        if (!lower) { A.y = -A.y; B.y = -B.y; }
        buf[n] = make_float2(A.x - B.y, A.y + B.x);
      }
    }
    __syncwarp();
    fft_line<L, 1, P>(buf, 1, lane, s_tw, active);
    if (active) {
      for (int n = lane; n < L; n += P) {
        const float2 z = buf[n];
        const long ia = ra * L + n;
        const float va = z.x * inv_sd;
        if (peak[ia] < va) { peak[ia] = va; angle[ia] = angle_id; }
        if (has_b) {
          const long ib = rb * L + n;
          const float vb = z.y * inv_sd;
          if (peak[ib] < vb) { peak[ib] = vb; angle[ib] = angle_id; }
        }
      }
    }
    __syncwarp();
  }
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
  const int grid = (int)std::max(1L, std::min((npairs + TEAMS - 1) / TEAMS, 8L * device_sm_count()));
  k_ts_c2r_mip<L, P><<<grid, TEAMS * P, 0, st>>>(in, nrows, stats, nvox, angle_id, peak, angle, tw);
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

}  // namespace emc

struct emc_tsearch_s {
  int nx, ny, nz;
  float2* T = nullptr;      // tomogram spectrum with the phase ramp
  float2* G = nullptr;      // template spectrum / product
  float2* S = nullptr;      // C2R scratch
  float* slab = nullptr;    // t real planes of the placed template
  int slab_t = 0;
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
  if (h->slab_t != t) {
    if (h->slab) cudaFree(h->slab);
    h->slab = nullptr;
    EMC_CUDA(cudaMalloc(&h->slab, sizeof(float) * (size_t)t * ny * nx));
    h->slab_t = t;
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
    // 1. rotated template into its t planes
    emc::k_ts_place<<<dim3((nx + 127) / 128, ny, t), 128, 0, st>>>(d_template, g, h->slab);
    EMC_LAUNCH_CHECK();
    // 2. pruned forward transform: x rows and y columns of the t planes, then z over all planes
    float2* Gp = h->G + (size_t)g.pl[2] * ny * nxh;
    EMC_TRY(emc::launch_rows_r2c(nx, h->slab, nx, Gp, nxh, (long)t * ny, st));
    EMC_TRY(emc::launch_cols(ny, -1, Gp, Gp, nxh, nxh, t, (long)ny * nxh, st));
    emc::k_ts_zero_planes<<<blocks, 256, 0, st>>>(h->G, g);
    EMC_LAUNCH_CHECK();
    EMC_TRY(emc::launch_cols(nz, -1, h->G, h->G, (long)ny * nxh, (long)ny * nxh, 1, (long)nz * ny * nxh, st));
    // 3. X = T conj(G) and its statistics
    EMC_CUDA(cudaMemsetAsync(h->stats, 0, 2 * sizeof(double), st));
    emc::k_ts_multiply<<<blocks, 256, 0, st>>>(h->T, h->G, g, h->stats);
    EMC_LAUNCH_CHECK();
    // 4. inverse z and y, then C2R along x fused with std normalisation and the MIP update
    EMC_TRY(emc::launch_cols(nz, 1, h->G, h->S, (long)ny * nxh, (long)ny * nxh, 1, (long)nz * ny * nxh, st));
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
  cudaFree(h->slab);
  cudaFree(h->stats);
  delete h;
  return EMC_OK;
}

}  // extern "C"
