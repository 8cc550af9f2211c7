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

// cos / sin(2 pi j / R) for the odd prime radices 5, 7 and 13 (exact values rounded to float).
__host__ __device__ constexpr float prime_cos(int R, int j) {
  return R == 5 ? (j == 0 ? 1.f : j == 1 ? 3.09016994374947451e-01f : j == 2 ? -8.09016994374947340e-01f
                 : j == 3 ? -8.09016994374947562e-01f : 3.09016994374947229e-01f)
       : R == 7 ? (j == 0 ? 1.f : j == 1 ? 6.23489801858733594e-01f : j == 2 ? -2.22520933956314337e-01f
                 : j == 3 ? -9.00968867902419035e-01f : j == 4 ? -9.00968867902419146e-01f
                 : j == 5 ? -2.22520933956314587e-01f : 6.23489801858733372e-01f)
                : (j == 0 ? 1.f : j == 1 ? 8.85456025653209911e-01f : j == 2 ? 5.68064746731155923e-01f
                 : j == 3 ? 1.20536680255323006e-01f : j == 4 ? -3.54604887042535455e-01f
                 : j == 5 ? -7.48510748171101192e-01f : j == 6 ? -9.70941817426052012e-01f
                 : j == 7 ? -9.70941817426052123e-01f : j == 8 ? -7.48510748171101303e-01f
                 : j == 9 ? -3.54604887042535899e-01f : j == 10 ? 1.20536680255323200e-01f
                 : j == 11 ? 5.68064746731154813e-01f : 8.85456025653210022e-01f);
}
__host__ __device__ constexpr float prime_sin(int R, int j) {
  return R == 5 ? (j == 0 ? 0.f : j == 1 ? 9.51056516295153531e-01f : j == 2 ? 5.87785252292473248e-01f
                 : j == 3 ? -5.87785252292473026e-01f : -9.51056516295153642e-01f)
       : R == 7 ? (j == 0 ? 0.f : j == 1 ? 7.81831482468029804e-01f : j == 2 ? 9.74927912181823619e-01f
                 : j == 3 ? 4.33883739117558231e-01f : j == 4 ? -4.33883739117558009e-01f
                 : j == 5 ? -9.74927912181823619e-01f : -7.81831482468029915e-01f)
                : (j == 0 ? 0.f : j == 1 ? 4.64723172043768507e-01f : j == 2 ? 8.22983865893656352e-01f
                 : j == 3 ? 9.92708874098053973e-01f : j == 4 ? 9.35016242685414833e-01f
                 : j == 5 ? 6.63122658240795193e-01f : j == 6 ? 2.39315664287557683e-01f
                 : j == 7 ? -2.39315664287557434e-01f : j == 8 ? -6.63122658240794971e-01f
                 : j == 9 ? -9.35016242685414722e-01f : j == 10 ? -9.92708874098053973e-01f
                 : j == 11 ? -8.22983865893657018e-01f : -4.64723172043768396e-01f);
}

// Odd prime radix: pairs (r, R-r) share the cosine term, X_q = x0 + sum_r [(x_r + x_{R-r}) cos
// + i SIGN (x_r - x_{R-r}) sin] with the angle 2 pi (q r mod R) / R.
template <int R, int SIGN>
struct DftPrime {
  static __host__ __device__ __forceinline__ void run(float2* v) {
    constexpr int H = (R - 1) / 2;
    float2 t1[H], t2[H];
#pragma unroll
    for (int r = 1; r <= H; ++r) {
      t1[r - 1] = cadd(v[r], v[R - r]);
      t2[r - 1] = csub(v[r], v[R - r]);
    }
    const float2 x0 = v[0];
    float2 s0 = x0;
#pragma unroll
    for (int r = 0; r < H; ++r) s0 = cadd(s0, t1[r]);
#pragma unroll
    for (int q = 1; q < R; ++q) {
      float2 acc = x0;
#pragma unroll
      for (int r = 1; r <= H; ++r) {
        const float c = prime_cos(R, (q * r) % R), s = (float)SIGN * prime_sin(R, (q * r) % R);
        acc.x = fmaf(t1[r - 1].x, c, fmaf(-t2[r - 1].y, s, acc.x));
        acc.y = fmaf(t1[r - 1].y, c, fmaf(t2[r - 1].x, s, acc.y));
      }
      v[q] = acc;
    }
    v[0] = s0;
  }
};
template <int SIGN> struct Dft<5, SIGN> : DftPrime<5, SIGN> {};
template <int SIGN> struct Dft<7, SIGN> : DftPrime<7, SIGN> {};
template <int SIGN> struct Dft<13, SIGN> : DftPrime<13, SIGN> {};

// ---------------------------------------------------------------- plans
// Generic plan for lengths without an explicit entry: radix-8 stages for the power of two (a 4
// or a 2 closes it), then 3s, 5s, 7s and 13s.  1 past the last stage, 0 for another prime factor.
__host__ __device__ constexpr int next_radix(int rem) {
  return rem % 8 == 0 ? 8 : rem % 4 == 0 ? 4 : rem % 2 == 0 ? 2 : rem % 3 == 0 ? 3 : rem % 5 == 0 ? 5
       : rem % 7 == 0 ? 7 : rem % 13 == 0 ? 13 : 0;
}
__host__ __device__ constexpr int radix_seq_rem(int rem, int s) {
  return rem == 1 ? 1 : next_radix(rem) == 0 ? 0 : s == 0 ? next_radix(rem) : radix_seq_rem(rem / next_radix(rem), s - 1);
}
__host__ __device__ constexpr int radix_seq(int L, int s) { return L < 2 ? 0 : radix_seq_rem(L, s); }

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
       // the remaining "nextBest" FFT sizes of coordinates/BH_multi_iterator.m:3-5 (factors 5, 7, 13)
       : radix_seq(L, s);
}

// Largest radix of a plan; used to pick a team size.
__host__ __device__ constexpr int max_radix(int L, int s = 0) {
  return radix_of(L, s) <= 1 ? 1
         : (radix_of(L, s) > max_radix(L, s + 1) ? radix_of(L, s) : max_radix(L, s + 1));
}
// Complex values a lane of a P-lane team holds in the largest stage of a length-L line.
__host__ __device__ constexpr int stage_values(int L, int P, int s = 0) {
  return radix_of(L, s) <= 1 ? 0
         : ((L / radix_of(L, s) + P - 1) / P) * radix_of(L, s) > stage_values(L, P, s + 1)
             ? ((L / radix_of(L, s) + P - 1) / P) * radix_of(L, s)
             : stage_values(L, P, s + 1);
}
__host__ __device__ constexpr int min_butterflies(int L) { return radix_of(L, 0) == 0 ? 0 : L / max_radix(L); }

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
// Physical slot of line element i.  With PAD, one spare slot follows every 8 elements: the
// radix-8 first stage writes elements 8j + r, which without the gap would put the 8 lanes of a
// team on 2 shared-memory banks.  padded_len(L) slots hold a padded line.
// PAD = 2 leaves the gap after every 16 elements instead, for lines whose first radix is 16
// (elements 16 j + r).
template <int PAD>
__host__ __device__ __forceinline__ constexpr int lpos(int i) {
  return PAD == 0 ? i : (PAD == 1 ? i + (i >> 3) : i + (i >> 4));
}
__host__ __device__ constexpr int padded_len(int L, int pad = 1) {
  return pad == 0 ? L : (pad == 1 ? L + L / 8 : L + L / 16);
}
// The padding that spreads the first stage's writes of a length-L line over the banks.  512
// (8 x 8 x 8) and 192 (8 x 8 x 3) also take the 16-element gap: their later stages read with
// strides of 64, where the 8-element gap leaves half-warps two or three ways on one bank (a
// half-warp model of the stage accesses gives 1.17 / 1.18 times the conflict-free wavefront
// count against 1.67 / 1.45 with the 8-element gap).
__host__ __device__ constexpr int line_pad(int L) {
  return radix_of(L, 0) >= 16 || L == 512 || L == 192 ? 2 : 1;
}

// Per-lane twiddles of stage S (NS = product of the earlier radices), kept in registers.  Lane
// `lane` of a team always handles butterflies j = lane + b P, whose twiddle exponents depend on
// k = j mod NS only -- not on which line the team transforms -- so a team can load them once
// and reuse them for every line.  Stages whose cache would exceed kTwCacheMax complex values
// (or that need no twiddles) read the shared-memory table instead.  The cache holds forward
// twiddles; inverse stages use their conjugates.
constexpr int kTwCacheMax = 8;

template <int L, int P, int S, int NS>
struct StageTw {
  static constexpr int R = radix_of(L, S);
  static constexpr int NB = L / R;
  static constexpr int PER = (NB + P - 1) / P;
  static constexpr bool kOn = NS > 1 && PER * (R - 1) <= kTwCacheMax;
  float2 w[kOn ? PER : 1][kOn ? R - 1 : 1];
  __device__ __forceinline__ void init(const float2* tw, int lane) {
    if constexpr (kOn) {
#pragma unroll
      for (int b = 0; b < PER; ++b) {
        const int k = (lane + b * P) % NS;
#pragma unroll
        for (int r = 1; r < R; ++r) w[b][r - 1] = tw[(r * k * (L / (NS * R))) % L];
      }
    }
  }
};

template <int L, int P, int S, int NS>
struct TwChain {
  StageTw<L, P, S, NS> st;
  TwChain<L, P, S + 1, NS * radix_of(L, S)> next;
  __device__ __forceinline__ void init(const float2* tw, int lane) {
    st.init(tw, lane);
    next.init(tw, lane);
  }
};
template <int L, int P, int S>
struct TwChain<L, P, S, L> {
  __device__ __forceinline__ void init(const float2*, int) {}
};

// Register twiddles of every stage of a length-L line transformed by teams of P lanes.
template <int L, int P = team_size(L)>
using LineTw = TwChain<L, P, 0, 1>;

// One Stockham stage of radix R on a line of length L (cache: optional register twiddles).
template <int L, int R, int NS, int SIGN, int P, int PAD, int S>
__device__ __forceinline__ void stockham_stage(float2* buf, int stride, int lane, const float2* tw,
                                               bool active, const StageTw<L, P, S, NS>* cache) {
  constexpr int NB = L / R;
  constexpr int PER = (NB + P - 1) / P;
  float2 v[PER][R];
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int j = lane + b * P;
    if (active && (PER * P == NB || j < NB)) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = buf[lpos<PAD>(j + r * NB) * stride];
    }
  }
  __syncwarp();
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int j = lane + b * P;
    if (active && (PER * P == NB || j < NB)) {
      const int k = j % NS;
      if constexpr (NS > 1) {
        if constexpr (StageTw<L, P, S, NS>::kOn) {
          if (cache) {
#pragma unroll
            for (int r = 1; r < R; ++r)
              v[b][r] = SIGN < 0 ? cmul(v[b][r], cache->w[b][r - 1]) : cmulc(v[b][r], cache->w[b][r - 1]);
          } else {
#pragma unroll
            for (int r = 1; r < R; ++r) v[b][r] = cmul(v[b][r], twiddle<SIGN>(tw, (r * k * (L / (NS * R))) % L));
          }
        } else {
#pragma unroll
          for (int r = 1; r < R; ++r) v[b][r] = cmul(v[b][r], twiddle<SIGN>(tw, (r * k * (L / (NS * R))) % L));
        }
      }
      Dft<R, SIGN>::run(v[b]);
      const int idx = (j / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) buf[lpos<PAD>(idx + r * NS) * stride] = v[b][r];
    }
  }
  __syncwarp();
}

template <int L, int SIGN, int P, int PAD, int S, int NS>
struct StageChain {
  static __device__ __forceinline__ void run(float2* buf, int stride, int lane, const float2* tw, bool active,
                                             const TwChain<L, P, S, NS>* tc) {
    constexpr int R = radix_of(L, S);
    stockham_stage<L, R, NS, SIGN, P, PAD, S>(buf, stride, lane, tw, active, tc ? &tc->st : nullptr);
    StageChain<L, SIGN, P, PAD, S + 1, NS * R>::run(buf, stride, lane, tw, active, tc ? &tc->next : nullptr);
  }
};
// terminate when the sub-transform length reaches L
template <int L, int SIGN, int P, int PAD, int S>
struct StageChain<L, SIGN, P, PAD, S, L> {
  static __device__ __forceinline__ void run(float2*, int, int, const float2*, bool, const TwChain<L, P, S, L>*) {}
};
// Stages S .. LAST-1 only (NS = product of the radices before S).
template <int L, int SIGN, int P, int PAD, int S, int NS, int LAST>
struct ForwardMidStages {
  static __device__ __forceinline__ void run(float2* buf, int stride, int lane, const float2* tw, bool active,
                                             const TwChain<L, P, S, NS>* tc) {
    if constexpr (S < LAST) {
      constexpr int R = radix_of(L, S);
      stockham_stage<L, R, NS, SIGN, P, PAD, S>(buf, stride, lane, tw, active, tc ? &tc->st : nullptr);
      ForwardMidStages<L, SIGN, P, PAD, S + 1, NS * R, LAST>::run(buf, stride, lane, tw, active,
                                                                 tc ? &tc->next : nullptr);
    }
  }
};

// First stage (NS = 1, no twiddles) with its inputs produced by ld(i) -- element i of the line
// -- instead of loaded from the buffer, so a caller that builds the line (packing two real rows,
// Hermitian extension) skips one shared-memory round trip.
template <int L, int R, int SIGN, int P, int PAD, class Ld>
__device__ __forceinline__ void stockham_first_stage_in(const Ld& ld, float2* buf, int stride, int lane, bool active) {
  constexpr int NB = L / R;
  constexpr int PER = (NB + P - 1) / P;
  float2 v[PER][R];
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int j = lane + b * P;
    if (active && (PER * P == NB || j < NB)) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = ld(j + r * NB);
      Dft<R, SIGN>::run(v[b]);
#pragma unroll
      for (int r = 0; r < R; ++r) buf[lpos<PAD>(j * R + r) * stride] = v[b][r];
    }
  }
  __syncwarp();
}

// In-place complex FFT of one line held by a team of P lanes.  Element i lives at
// buf[lpos<PAD>(i) * stride].  tc (optional) holds the team lane's register twiddles.
template <int L, int SIGN, int P = team_size(L), int PAD = 0>
__device__ __forceinline__ void fft_line(float2* buf, int stride, int lane, const float2* tw, bool active,
                                         const LineTw<L, P>* tc = nullptr) {
  static_assert(radix_of(L, 0) != 0, "unsupported FFT length");
  static_assert(P >= 1 && P <= 32 && (32 % P) == 0, "team must divide a warp");
  StageChain<L, SIGN, P, PAD, 0, 1>::run(buf, stride, lane, tw, active, tc);
}

// FFT of a line whose elements come from ld(i) (see stockham_first_stage_in); the result is left
// in buf like fft_line's.
template <int L, int SIGN, int P = team_size(L), int PAD = 0, class Ld>
__device__ __forceinline__ void fft_line_in(const Ld& ld, float2* buf, int stride, int lane, const float2* tw,
                                            bool active, const LineTw<L, P>* tc = nullptr) {
  static_assert(radix_of(L, 0) != 0, "unsupported FFT length");
  constexpr int R0 = radix_of(L, 0);
  stockham_first_stage_in<L, R0, SIGN, P, PAD>(ld, buf, stride, lane, active);
  StageChain<L, SIGN, P, PAD, 1, R0>::run(buf, stride, lane, tw, active, tc ? &tc->next : nullptr);
}

// Number of Stockham stages of a length-L plan and the product of the radices before stage s.
__host__ __device__ constexpr int n_stages(int L, int s = 0);
__host__ __device__ constexpr int radix_product(int L, int s);

// The last Stockham stage of a length-L plan for teams of P lanes: radix RL, NSL = L / RL
// butterflies (the product of the earlier radices), PER butterflies per lane.
template <int L, int P>
struct LastStage {
  static constexpr int S = n_stages(L) - 1;
  static constexpr int RL = radix_of(L, S);
  static constexpr int NSL = L / RL;
  static constexpr int PER = (NSL + P - 1) / P;
};

// Register twiddles of stage S of a chain (nullptr when the chain holds none for it).
template <int S, int L, int P, int S0, int NS>
__device__ __forceinline__ const StageTw<L, P, S, radix_product(L, S)>* stage_tw(const TwChain<L, P, S0, NS>* tc) {
  if constexpr (S0 == S) {
    return tc ? &tc->st : nullptr;
  } else {
    return stage_tw<S>(tc ? &tc->next : (const TwChain<L, P, S0 + 1, NS * radix_of(L, S0)>*)nullptr);
  }
}

// FFT of a line whose elements come from ld(i), like fft_line_in, with the last stage left in
// registers: on return v[b][r] holds element (lane + b P) + NSL r of the transform for every
// butterfly lane + b P < NSL of an active lane (LastStage<L, P>); buf holds the earlier stages'
// scratch.  The caller synchronises the team before buf is written again.
template <int L, int SIGN, int P, int PAD, class Ld>
__device__ __forceinline__ void fft_line_in_regs(const Ld& ld, float2* buf, int stride, int lane, const float2* tw,
                                                 bool active, const LineTw<L, P>* tc,
                                                 float2 (&v)[LastStage<L, P>::PER][LastStage<L, P>::RL]) {
  using LS = LastStage<L, P>;
  constexpr int R0 = radix_of(L, 0);
  static_assert(LS::S >= 1, "at least two stages");
  stockham_first_stage_in<L, R0, SIGN, P, PAD>(ld, buf, stride, lane, active);
  if constexpr (LS::S > 1) {
    // stages 1 .. S-1 in shared memory
    ForwardMidStages<L, SIGN, P, PAD, 1, R0, LS::S>::run(buf, stride, lane, tw, active, tc ? &tc->next : nullptr);
  }
  const auto* cache = stage_tw<LS::S>(tc);
#pragma unroll
  for (int b = 0; b < LS::PER; ++b) {
    const int j = lane + b * P;
    if (active && (LS::PER * P == LS::NSL || j < LS::NSL)) {
#pragma unroll
      for (int r = 0; r < LS::RL; ++r) v[b][r] = buf[lpos<PAD>(j + r * LS::NSL) * stride];
      if constexpr (StageTw<L, P, LS::S, LS::NSL>::kOn) {
        if (cache) {
#pragma unroll
          for (int r = 1; r < LS::RL; ++r)
            v[b][r] = SIGN < 0 ? cmul(v[b][r], cache->w[b][r - 1]) : cmulc(v[b][r], cache->w[b][r - 1]);
        } else {
#pragma unroll
          for (int r = 1; r < LS::RL; ++r) v[b][r] = cmul(v[b][r], twiddle<SIGN>(tw, (r * j) % L));
        }
      } else {
#pragma unroll
        for (int r = 1; r < LS::RL; ++r) v[b][r] = cmul(v[b][r], twiddle<SIGN>(tw, (r * j) % L));
      }
      Dft<LS::RL, SIGN>::run(v[b]);
    }
  }
}
__host__ __device__ constexpr int n_stages(int L, int s) { return radix_of(L, s) <= 1 ? s : n_stages(L, s + 1); }
__host__ __device__ constexpr int radix_product(int L, int s) { return s == 0 ? 1 : radix_of(L, s - 1) * radix_product(L, s - 1); }

// Forward stages S .. LAST-1 of a length-L line (NS = product of the radices before S).
template <int L, int P, int PAD, int S, int LAST>
struct ForwardStages {
  static __device__ __forceinline__ void run(float2* buf, int stride, int lane, const float2* tw, bool active) {
    if constexpr (S < LAST) {
      stockham_stage<L, radix_of(L, S), radix_product(L, S), -1, P, PAD, S>(buf, stride, lane, tw, active, nullptr);
      ForwardStages<L, P, PAD, S + 1, LAST>::run(buf, stride, lane, tw, active);
    }
  }
};
// Inverse stages with the forward radices taken in reverse order, from forward stage S down to 0
// (NS = product of the radices already applied).  A mixed-radix transform may take its radices in
// any order; this one starts with the forward plan's last radix.
template <int L, int P, int PAD, int S, int NS>
struct InverseStagesReversed {
  static __device__ __forceinline__ void run(float2* buf, int stride, int lane, const float2* tw, bool active) {
    if constexpr (S >= 0) {
      stockham_stage<L, radix_of(L, S), NS, 1, P, PAD, S>(buf, stride, lane, tw, active, nullptr);
      InverseStagesReversed<L, P, PAD, S - 1, NS * radix_of(L, S)>::run(buf, stride, lane, tw, active);
    }
  }
};
template <int L, int P, int PAD, int NS>
struct InverseStagesReversed<L, P, PAD, -1, NS> {
  static __device__ __forceinline__ void run(float2*, int, int, const float2*, bool) {}
};

// Forward transform, elementwise product, inverse transform of one line, with the product formed in
// registers.  The forward transform's stages but the last run in shared memory; its last stage
// (radix RL, NS = L / RL) leaves lane j of the team holding, for each of its butterflies
// j' = j + b P, the elements z = j' + (L / RL) r -- the elements the inverse transform's first stage
// needs when the inverse takes the radices in reverse order (radix RL first, NB = L / RL).  So
// mul(z, X(z)) -> Y(z) is applied to those registers, the inverse's first stage runs on them and its
// remaining stages in shared memory: two shared-memory passes over the line fewer than
// fft_line(-1), a separate product and fft_line(+1).  Element i of the line lives at
// buf[lpos<PAD>(i) * stride]; the result (unnormalised) is left there in natural order.
template <int L, int P, int PAD, class Mul>
__device__ __forceinline__ void fft_line_fwd_mul_inv(float2* buf, int stride, int lane, const float2* tw, bool active,
                                                     Mul&& mul) {
  constexpr int LAST = n_stages(L) - 1;
  constexpr int RL = radix_of(L, LAST), NSL = L / RL, PER = (NSL + P - 1) / P;
  ForwardStages<L, P, PAD, 0, LAST>::run(buf, stride, lane, tw, active);
  float2 v[PER][RL];
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int j = lane + b * P;
    if (active && (PER * P == NSL || j < NSL)) {
#pragma unroll
      for (int r = 0; r < RL; ++r) v[b][r] = buf[lpos<PAD>(j + r * NSL) * stride];
      if constexpr (LAST > 0) {
#pragma unroll
        for (int r = 1; r < RL; ++r) v[b][r] = cmul(v[b][r], twiddle<-1>(tw, (r * j) % L));
      }
      Dft<RL, -1>::run(v[b]);
#pragma unroll
      for (int r = 0; r < RL; ++r) v[b][r] = mul(j + NSL * r, v[b][r]);
      Dft<RL, 1>::run(v[b]);
    }
  }
  __syncwarp();  // every lane has read the line before any writes it
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int j = lane + b * P;
    if (active && (PER * P == NSL || j < NSL)) {
#pragma unroll
      for (int r = 0; r < RL; ++r) buf[lpos<PAD>(j * RL + r) * stride] = v[b][r];
    }
  }
  __syncwarp();
  InverseStagesReversed<L, P, PAD, LAST - 1, RL>::run(buf, stride, lane, tw, active);
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
