// fft_passes.cuh -- generic single-axis FFT passes over global memory.
//
// These are the building blocks of the standalone R2C / C2R transform (the mexFFT
// replacement), of the particle-spectrum preparation and of the large-volume
// template search.  The fused orientation-search kernels use the same line FFT
// but keep the data on chip between axes.
#pragma once
#include "common.cuh"

namespace emc {

// ----------------------------------------------------------------- rows, R2C
// nrows real rows of length L (pitch in_pitch floats) -> complex rows of length
// L/2+1 (pitch out_pitch float2).  Two rows share one complex FFT: z = a + i b.
// Teams per CTA of the row kernels: at most 256 threads and ~32 KB of line buffers.
// Line buffers hold padded lines (lpos<line_pad(L)>, see fft.cuh) against bank conflicts.
__host__ __device__ constexpr int row_line_len(int L) { return padded_len(L, line_pad(L)) + 1; }
__host__ __device__ constexpr int rows_teams(int L, int P) {
  return (256 / P) < (4096 / row_line_len(L)) ? (256 / P)
                                               : ((4096 / row_line_len(L)) > 0 ? (4096 / row_line_len(L)) : 1);
}

template <int L, int P>
__global__ void __launch_bounds__(256) k_rows_r2c(const float* __restrict__ in, long in_pitch,
                                                  float2* __restrict__ out, long out_pitch, long nrows,
                                                  const float2* __restrict__ g_tw) {
  constexpr int TEAMS = rows_teams(L, P);
  constexpr int PAD = line_pad(L);
  __shared__ float2 s_tw[L];
  __shared__ float2 s_line[TEAMS][row_line_len(L)];
  load_twiddles<L>(s_tw, g_tw);
  __syncthreads();
  const int team = threadIdx.x / P, lane = threadIdx.x % P;
  const long npairs = (nrows + 1) / 2;
  for (long pair0 = (long)blockIdx.x * TEAMS; pair0 < npairs; pair0 += (long)gridDim.x * TEAMS) {
    const long pair = pair0 + team;
    const bool active = pair < npairs;
    const long ra = 2 * pair, rb = 2 * pair + 1;
    const bool has_b = rb < nrows;
    float2* buf = s_line[team];
    const float* a = in + ra * in_pitch;
    const float* b = in + rb * in_pitch;
    fft_line_in<L, -1, P, PAD>([&](int n) { return make_float2(__ldg(a + n), has_b ? __ldg(b + n) : 0.f); }, buf,
                               1, lane, s_tw, active);
    if (active) {
      float2* oa = out + ra * out_pitch;
      float2* ob = out + rb * out_pitch;
      for (int k = lane; k <= L / 2; k += P) {
        const float2 zk = buf[lpos<PAD>(k)], zm = buf[lpos<PAD>((L - k) % L)];
        oa[k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        if (has_b) ob[k] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
      }
    }
    __syncwarp();
  }
}

// ----------------------------------------------------------------- rows, C2R
// complex rows of length L/2+1 -> real rows of length L (unnormalised inverse).
// The imaginary parts of the k = 0 and k = L/2 terms are ignored (real-part
// semantics of a Hermitian inverse).
template <int L, int P>
__global__ void __launch_bounds__(256) k_rows_c2r(const float2* __restrict__ in, long in_pitch,
                                                  float* __restrict__ out, long out_pitch, long nrows,
                                                  const float2* __restrict__ g_tw) {
  constexpr int TEAMS = rows_teams(L, P);
  constexpr int PAD = line_pad(L);
  __shared__ float2 s_tw[L];
  __shared__ float2 s_line[TEAMS][row_line_len(L)];
  load_twiddles<L>(s_tw, g_tw);
  __syncthreads();
  const int team = threadIdx.x / P, lane = threadIdx.x % P;
  const long npairs = (nrows + 1) / 2;
  for (long pair0 = (long)blockIdx.x * TEAMS; pair0 < npairs; pair0 += (long)gridDim.x * TEAMS) {
    const long pair = pair0 + team;
    const bool active = pair < npairs;
    const long ra = 2 * pair, rb = 2 * pair + 1;
    const bool has_b = rb < nrows;
    float2* buf = s_line[team];
    const float2* a = in + ra * in_pitch;
    const float2* b = in + rb * in_pitch;
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
      float* oa = out + ra * out_pitch;
      float* ob = out + rb * out_pitch;
      for (int n = lane; n < L; n += P) {
        const float2 z = buf[lpos<PAD>(n)];
        oa[n] = z.x;
        if (has_b) ob[n] = z.y;
      }
    }
    __syncwarp();
  }
}

// ----------------------------------------------------------------- strided columns
// Complex lines along a strided axis: element n of line (o, i) lives at
// base + o*outer_pitch + i + n*stride, for i in [0, inner), o in [0, outer).
// A unit of work is a tile of T consecutive i of one o; in == out is allowed (units are disjoint).
// Persistent CTAs walk the units with a stride of gridDim.x and double-buffer them in shared
// memory: the cp.async copies of the next tile are in flight while the current tile is
// transformed and written back, so the loads of a one-CTA-per-SM kernel overlap its FFT.
template <int L, int SIGN, int P, int T>
__global__ void __launch_bounds__(P * T) k_cols(const float2* __restrict__ in, float2* __restrict__ out,
                                                long stride, long inner, long outer, long outer_pitch,
                                                const float2* __restrict__ g_tw) {
  extern __shared__ float2 smem[];
  constexpr int TP = T + 1;
  constexpr int PAD = line_pad(L);
  constexpr int TILE = padded_len(L, PAD) * TP;  // element n of line t at lpos<PAD>(n) * TP + t
  float2* s_tw = smem;
  float2* tiles = smem + L;  // [2][TILE]
  load_twiddles<L>(s_tw, g_tw);
  const long ntile = (inner + T - 1) / T;
  const long units = ntile * outer;
  constexpr int NT = P * T;
  const int team = threadIdx.x / P, lane = threadIdx.x % P;
  auto issue = [&](long u, float2* tile) {
    const long o = u / ntile, i0 = (u % ntile) * T;
    const float2* src = in + o * outer_pitch + i0;
#pragma unroll 4
    for (int idx = threadIdx.x; idx < L * T; idx += NT) {
      const int n = idx / T, t = idx % T;
      if (i0 + t < inner) cp_async8(tile + lpos<PAD>(n) * TP + t, src + (long)n * stride + t);
    }
    cp_async_commit();
  };
  long u = blockIdx.x;
  if (u < units) issue(u, tiles);
  int cur = 0;
  for (; u < units; u += gridDim.x) {
    const long un = u + gridDim.x;
    if (un < units) {
      issue(un, tiles + (cur ^ 1) * TILE);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();  // tile `cur` (and the twiddles) visible to every thread
    float2* tile = tiles + cur * TILE;
    const long o = u / ntile, i0 = (u % ntile) * T;
    fft_line<L, SIGN, P, PAD>(tile + team, TP, lane, s_tw, i0 + team < inner);
    __syncthreads();
    float2* dst = out + o * outer_pitch + i0;
    for (int idx = threadIdx.x; idx < L * T; idx += NT) {
      const int n = idx / T, t = idx % T;
      if (i0 + t < inner) dst[(long)n * stride + t] = tile[lpos<PAD>(n) * TP + t];
    }
    __syncthreads();  // tile `cur` has been read; the next iteration's copies land in it
    cur ^= 1;
  }
}

template <int L>
struct ColsCfg {
  static constexpr int P = team_size(L);
  static constexpr int T = (512 / P) < 32 ? (512 / P) : 32;
  static constexpr size_t smem = sizeof(float2) * (L + 2 * (size_t)padded_len(L, line_pad(L)) * (T + 1));
};

// Host launchers (defined in fft_passes.cu); return EMC_OK or an error status.
emc_status launch_rows_r2c(int L, const float* in, long in_pitch, float2* out, long out_pitch, long nrows,
                           cudaStream_t st);
emc_status launch_rows_c2r(int L, const float2* in, long in_pitch, float* out, long out_pitch, long nrows,
                           cudaStream_t st);
emc_status launch_cols(int L, int sign, const float2* in, float2* out, long stride, long inner, long outer,
                       long outer_pitch, cudaStream_t st);

// Full 3-D R2C / C2R over a batch of volumes (x fastest).  c2r uses `scratch`
// ((nx/2+1)*ny*nz*batch float2) so that `in` is left untouched.
emc_status fft3_r2c(const float* in, float2* out, int nx, int ny, int nz, int batch, cudaStream_t st);
emc_status fft3_c2r(const float2* in, float* out, float2* scratch, int nx, int ny, int nz, int batch,
                    cudaStream_t st);

}  // namespace emc
