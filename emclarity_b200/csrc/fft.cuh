// fft.cuh -- hand-written FP32 FFT building blocks for sm_100a.
//
// A line of length L (L = 2^a 3^b) is transformed in place in shared memory by a
// "team" of P lanes of one warp (P divides 32).  Stages follow the Stockham
// autosort formulation with mixed radices {2,3,4,8,16}: each lane loads all the
// inputs of its butterflies into registers, the warp synchronises, then the lane
// applies twiddles, runs the radix-R DFT codelet in registers and stores.  With
// two or three stages per line, data crosses shared memory 2-3 times per axis.
//
// Sign convention: SIGN = -1 is the forward transform X_k = sum x_n e^{-2 pi i nk/L}
// (cuFFT / MATLAB fftn), SIGN = +1 the unnormalised inverse.
//
// Twiddles come from a per-length table tw[m] = exp(-2 pi i m / L), m in [0, L),
// computed on the host in double precision and rounded to float.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace emc {

__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// a * (SIGN * i)
template <int SIGN>
__host__ __device__ __forceinline__ float2 mul_si(float2 a) {
  return SIGN < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

// cos / sin of rational multiples of pi used inside the codelets (exact math constants).
#define EMC_SQRT1_2 0.70710678118654752440f
#define EMC_COS_PI8 0.92387953251128675613f
#define EMC_SIN_PI8 0.38268343236508977173f
#define EMC_SQRT3_2 0.86602540378443864676f

// ---------------------------------------------------------------- codelets
template <int R, int SIGN> struct Dft;

template <int SIGN> struct Dft<1, SIGN> {
  static __host__ __device__ __forceinline__ void run(float2*) {}
};

template <int SIGN> struct Dft<2, SIGN> {
  static __host__ __device__ __forceinline__ void run(float2* v) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <int SIGN> struct Dft<3, SIGN> {
  static __host__ __device__ __forceinline__ void run(float2* v) {
    float2 t1 = cadd(v[1], v[2]);
    float2 t2 = make_float2(fmaf(-0.5f, t1.x, v[0].x), fmaf(-0.5f, t1.y, v[0].y));
    float2 d = csub(v[1], v[2]);
    // i * SIGN * sqrt(3)/2 * d
    float2 t3 = mul_si<SIGN>(cscale(d, EMC_SQRT3_2));
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  }
};

template <int SIGN> struct Dft<4, SIGN> {
  static __host__ __device__ __forceinline__ void run(float2* v) {
    float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    float2 b0 = cadd(v[1], v[3]), b1 = mul_si<SIGN>(csub(v[1], v[3]));
    v[0] = cadd(a0, b0);
    v[2] = csub(a0, b0);
    v[1] = cadd(a1, b1);
    v[3] = csub(a1, b1);
  }
};

template <int SIGN> struct Dft<8, SIGN> {
  static __host__ __device__ __forceinline__ void run(float2* v) {
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, SIGN>::run(e);
    Dft<4, SIGN>::run(o);
    // w8^k = exp(SIGN 2 pi i k / 8)
    float2 o1 = cscale(make_float2(o[1].x - (float)SIGN * o[1].y, o[1].y + (float)SIGN * o[1].x), EMC_SQRT1_2);
    float2 o2 = mul_si<SIGN>(o[2]);
    float2 o3 = cscale(make_float2(-o[3].x - (float)SIGN * o[3].y, -o[3].y + (float)SIGN * o[3].x), EMC_SQRT1_2);
    v[0] = cadd(e[0], o[0]); v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);   v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);   v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);   v[7] = csub(e[3], o3);
  }
};

template <int SIGN> struct Dft<16, SIGN> {
  static __host__ __device__ __forceinline__ void run(float2* v) {
    float2 e[8], o[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) { e[i] = v[2 * i]; o[i] = v[2 * i + 1]; }
    Dft<8, SIGN>::run(e);
    Dft<8, SIGN>::run(o);
    const float s = (float)SIGN;
    // w16^k = cos(2 pi k/16) + i SIGN sin(2 pi k/16)
    const float2 w[8] = {
        make_float2(1.f, 0.f),
        make_float2(EMC_COS_PI8, s * EMC_SIN_PI8),
        make_float2(EMC_SQRT1_2, s * EMC_SQRT1_2),
        make_float2(EMC_SIN_PI8, s * EMC_COS_PI8),
        make_float2(0.f, s),
        make_float2(-EMC_SIN_PI8, s * EMC_COS_PI8),
        make_float2(-EMC_SQRT1_2, s * EMC_SQRT1_2),
        make_float2(-EMC_COS_PI8, s * EMC_SIN_PI8)};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      float2 t = (k == 0) ? o[0] : cmul(o[k], w[k]);
      v[k] = cadd(e[k], t);
      v[k + 8] = csub(e[k], t);
    }
  }
};

// ---------------------------------------------------------------- plans
// Radix sequence per supported length.  Stage s uses radix radix_of(L, s); 1 ends the plan.
__host__ __device__ constexpr int radix_of(int L, int s) {
  return L == 2   ? (s == 0 ? 2 : 1)
       : L == 3   ? (s == 0 ? 3 : 1)
       : L == 4   ? (s == 0 ? 4 : 1)
       : L == 6   ? (s == 0 ? 3 : s == 1 ? 2 : 1)
       : L == 8   ? (s == 0 ? 8 : 1)
       : L == 12  ? (s == 0 ? 4 : s == 1 ? 3 : 1)
       : L == 16  ? (s == 0 ? 16 : 1)
       : L == 24  ? (s == 0 ? 8 : s == 1 ? 3 : 1)
       : L == 32  ? (s == 0 ? 8 : s == 1 ? 4 : 1)
       : L == 48  ? (s == 0 ? 16 : s == 1 ? 3 : 1)
       : L == 64  ? (s == 0 ? 8 : s == 1 ? 8 : 1)
       : L == 96  ? (s == 0 ? 8 : s == 1 ? 4 : s == 2 ? 3 : 1)
       : L == 128 ? (s == 0 ? 16 : s == 1 ? 8 : 1)
       : L == 192 ? (s == 0 ? 8 : s == 1 ? 8 : s == 2 ? 3 : 1)
       : L == 256 ? (s == 0 ? 16 : s == 1 ? 16 : 1)
       : L == 384 ? (s == 0 ? 16 : s == 1 ? 8 : s == 2 ? 3 : 1)
       : L == 512 ? (s == 0 ? 8 : s == 1 ? 8 : s == 2 ? 8 : 1)
       : 0;
}

// Largest radix of a plan; used to pick a team size.
__host__ __device__ constexpr int min_butterflies(int L) {
  return (radix_of(L, 0) == 0) ? 0
         : (L / (radix_of(L, 0) > radix_of(L, 1) ? (radix_of(L, 0) > radix_of(L, 2) ? radix_of(L, 0) : radix_of(L, 2))
                                                 : (radix_of(L, 1) > radix_of(L, 2) ? radix_of(L, 1) : radix_of(L, 2))));
}

// Default team size: a power of two no larger than the smallest butterfly count, <= 32.
__host__ __device__ constexpr int team_size(int L) {
  return min_butterflies(L) >= 32 ? 32
       : min_butterflies(L) >= 16 ? 16
       : min_butterflies(L) >= 8  ? 8
       : min_butterflies(L) >= 4  ? 4
       : min_butterflies(L) >= 2  ? 2 : 1;
}

template <int SIGN>
__device__ __forceinline__ float2 twiddle(const float2* tw, int m) {
  float2 t = tw[m];
  return SIGN < 0 ? t : make_float2(t.x, -t.y);
}

// One Stockham stage of radix R on a line of length L; NS = product of earlier radices.
// buf: line base, elements at buf[i * stride].  Every lane of the warp must call this
// (inactive lanes pass active = false) because of the __syncwarp() calls.
template <int L, int R, int NS, int SIGN, int P>
__device__ __forceinline__ void stockham_stage(float2* buf, int stride, int lane, const float2* tw,
                                               bool active) {
  constexpr int NB = L / R;
  constexpr int PER = (NB + P - 1) / P;
  float2 v[PER][R];
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int j = lane + b * P;
    if (active && (PER * P == NB || j < NB)) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = buf[(j + r * NB) * stride];
    }
  }
  __syncwarp();
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int j = lane + b * P;
    if (active && (PER * P == NB || j < NB)) {
      const int k = j % NS;
      if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) v[b][r] = cmul(v[b][r], twiddle<SIGN>(tw, (r * k * (L / (NS * R))) % L));
      }
      Dft<R, SIGN>::run(v[b]);
      const int idx = (j / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) buf[(idx + r * NS) * stride] = v[b][r];
    }
  }
  __syncwarp();
}

template <int L, int SIGN, int P, int S, int NS>
struct StageChain {
  static __device__ __forceinline__ void run(float2* buf, int stride, int lane, const float2* tw, bool active) {
    constexpr int R = radix_of(L, S);
    stockham_stage<L, R, NS, SIGN, P>(buf, stride, lane, tw, active);
    StageChain<L, SIGN, P, S + 1, NS * R>::run(buf, stride, lane, tw, active);
  }
};
// terminate when the sub-transform length reaches L
template <int L, int SIGN, int P, int S>
struct StageChain<L, SIGN, P, S, L> {
  static __device__ __forceinline__ void run(float2*, int, int, const float2*, bool) {}
};

// In-place complex FFT of one line held by a team of P lanes.
template <int L, int SIGN, int P = team_size(L)>
__device__ __forceinline__ void fft_line(float2* buf, int stride, int lane, const float2* tw, bool active) {
  static_assert(radix_of(L, 0) != 0, "unsupported FFT length");
  static_assert(P >= 1 && P <= 32 && (32 % P) == 0, "team must divide a warp");
  StageChain<L, SIGN, P, 0, 1>::run(buf, stride, lane, tw, active);
}

// Loads the length-L twiddle table into shared memory (cooperatively, whole block).
template <int L>
__device__ __forceinline__ void load_twiddles(float2* s_tw, const float2* g_tw) {
  for (int i = threadIdx.x + threadIdx.y * blockDim.x; i < L; i += blockDim.x * blockDim.y) s_tw[i] = g_tw[i];
}

// Map a float to an unsigned key with the same order (for atomicMax-based argmax).
__device__ __forceinline__ uint32_t ordered_key(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ inline float key_to_float(uint32_t k) {
  uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}

}  // namespace emc
