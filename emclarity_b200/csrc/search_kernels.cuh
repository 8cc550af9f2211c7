// search_kernels.cuh -- the three fused passes of one CC evaluation (particle, orientation).
//
// Data flow per evaluation e (box n, half width nh = n/2+1, peak radius r, window w = 2r+1):
//   pass A  (CTA = G z-planes)   gather r = mask .* I(M (p - c - t) + c)  -> smem
//                                (no weight on the reference: FP64 sums of r and r^2, the
//                                DC-free energy by Parseval)
//                                R2C along x (two rows per complex FFT), FFT along y
//                                -> S1[e][ky][part][z][kx], one padded slab per (ky, column part)
//                                   in pass B's tile layout                (~n * n * nh c64)
//   pass B  (CTA = one ky row    slab in by one bulk copy; FFT along z, X = Q .* conj(wref .* R)
//            or half of one)     .* wdgMask, X(0) = 0, E_R = sum |wref .* R .* wdgMask|^2 when
//                                either weight is set (formed in registers between the
//                                transforms, fft_line_fwd_mul_inv), inverse FFT along z, keep the
//                                w output planes |sz| <= r
//                                -> S2[e][j][ky][kx], planes in pass C's tile layout  (~w * n * nh c64)
//   pass C  (CTA = one sz plane) inverse FFT along y, C2R along x for the w rows |sy| <= r,
//                                normalise by sqrt(E_R E_P), spherical peak mask,
//                                argmax -> atomicMax on a 64-bit (cc, -index) key
// The reference computes the whole map (BH_multi_xcf_Translational_2.m:35-38) and then
// masks it (BH_multi_xcf_Translational.m:33-42); only the masked window is evaluated here.
#pragma once
#include "interp.cuh"

namespace emc {

struct DevParticle {
  const float2* spec;  // Q = refWdg .* P, [z][y][kx]
  const float* wedge;  // wdgMask, the weight on the rotated reference, [z][y][kx] or null (= 1)
  double energy;       // E_P = sum |Q|^2
  double prior[9];     // column-major
  float shift[3];
  int ref;
  int box;
  int orient_begin;
  long eval_base;      // index of this particle's first (p, o) pair in the output order
};

struct DevRef {
  const void* data;    // n^3, float or bf16
  const float* mask;   // n^3 or null
  const float* wref;   // nh*n*n or null
  int n;
  int dtype;
  const void* cells;   // (n+1)^3 trilinear corner cells (see build_cells) or null
  const unsigned* mask_rows;  // per (z, y) row: lo | hi << 16, the x extent [lo, hi) of mask != 0, or null
};

// Trilinear corner cells: cell (i, j, k), i, j, k in [-1, n-1], holds the 8 voxels
// v(i+a, j+b, k+c), a, b, c in {0, 1}, in the order (000, 100, 010, 110, 001, 101, 011, 111),
// zero outside the volume.  One 32-byte (FP32) or 16-byte (BF16) vector load fetches every
// corner a trilinear sample needs, instead of eight scattered 4-byte loads.
template <typename T>
struct CellT;
template <>
struct CellT<float> {
  float4 lo, hi;
};
template <>
struct CellT<__nv_bfloat16> {
  uint4 v;
};

__device__ __forceinline__ void cell_values(const CellT<float>& c, float v[8]) {
  v[0] = c.lo.x; v[1] = c.lo.y; v[2] = c.lo.z; v[3] = c.lo.w;
  v[4] = c.hi.x; v[5] = c.hi.y; v[6] = c.hi.z; v[7] = c.hi.w;
}
__device__ __forceinline__ void cell_values(const CellT<__nv_bfloat16>& c, float v[8]) {
  const __nv_bfloat162* p = reinterpret_cast<const __nv_bfloat162*>(&c.v);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float2 f = __bfloat1622float2(p[i]);
    v[2 * i] = f.x;
    v[2 * i + 1] = f.y;
  }
}
// One 256-bit read-only load (sm_100): the whole 32-byte cell in a single request, so the cell's
// sector is looked up once instead of once per 16-byte half.  Cells are 32-byte aligned.
__device__ __forceinline__ CellT<float> load_cell(const CellT<float>* p) {
  CellT<float> c;
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(c.lo.x), "=f"(c.lo.y), "=f"(c.lo.z), "=f"(c.lo.w), "=f"(c.hi.x), "=f"(c.hi.y), "=f"(c.hi.z),
        "=f"(c.hi.w)
      : "l"(p));
  return c;
}
__device__ __forceinline__ CellT<__nv_bfloat16> load_cell(const CellT<__nv_bfloat16>* p) {
  CellT<__nv_bfloat16> c;
  c.v = __ldg(&p->v);
  return c;
}

// Cell index and fractions of sample point s; `valid` follows interpn (MODE 0: 0 <= s <= n-1)
// or the zero-border texture addressing (MODE 2: -1 < s < n).
template <int MODE>
__device__ __forceinline__ long cell_index(int n, float sx, float sy, float sz, float f[3], bool* valid) {
  const bool ok = MODE == EMC_INTERP_LINEAR_BORDER
                      ? (sx > -1.f && sy > -1.f && sz > -1.f && sx < (float)n && sy < (float)n && sz < (float)n)
                      : (sx >= 0.f && sy >= 0.f && sz >= 0.f && sx <= (float)(n - 1) && sy <= (float)(n - 1) &&
                         sz <= (float)(n - 1));
  const float fx0 = floorf(sx), fy0 = floorf(sy), fz0 = floorf(sz);
  const int x0 = max(-1, min((int)fx0, n - 1)), y0 = max(-1, min((int)fy0, n - 1)), z0 = max(-1, min((int)fz0, n - 1));
  f[0] = sx - (float)x0;
  f[1] = sy - (float)y0;
  f[2] = sz - (float)z0;
  *valid = ok;
  const long nc = n + 1;
  return ((long)(z0 + 1) * nc + (y0 + 1)) * nc + (x0 + 1);
}

// cell_index for the search gather: floor by a round-down conversion, 32-bit index arithmetic,
// and no clamping -- an invalid sample reads cell 0 and its value is discarded by the caller
// (`valid` false), so only in-range indices ever reach memory.
template <int MODE>
__device__ __forceinline__ unsigned cell_index_gather(int n, float sx, float sy, float sz, float f[3], bool& valid) {
  valid = MODE == EMC_INTERP_LINEAR_BORDER
              ? (sx > -1.f && sy > -1.f && sz > -1.f && sx < (float)n && sy < (float)n && sz < (float)n)
              : (sx >= 0.f && sy >= 0.f && sz >= 0.f && sx <= (float)(n - 1) && sy <= (float)(n - 1) &&
                 sz <= (float)(n - 1));
  const int x0 = __float2int_rd(sx), y0 = __float2int_rd(sy), z0 = __float2int_rd(sz);
  f[0] = sx - (float)x0;
  f[1] = sy - (float)y0;
  f[2] = sz - (float)z0;
  const unsigned nc = (unsigned)n + 1u;
  const unsigned idx = ((unsigned)(z0 + 1) * nc + (unsigned)(y0 + 1)) * nc + (unsigned)(x0 + 1);
  return valid ? idx : 0u;
}

// Same interpolation order as sample_linear, so both paths give identical results.
__device__ __forceinline__ float cell_trilinear(const float v[8], const float f[3]) {
  const float c00 = fmaf(f[0], v[1] - v[0], v[0]), c10 = fmaf(f[0], v[3] - v[2], v[2]);
  const float c01 = fmaf(f[0], v[5] - v[4], v[4]), c11 = fmaf(f[0], v[7] - v[6], v[6]);
  const float c0 = fmaf(f[1], c10 - c00, c00), c1 = fmaf(f[1], c11 - c01, c01);
  return fmaf(f[2], c1 - c0, c0);
}

// Builds the corner cells of an n^3 FP32 volume, stored as T.
template <typename T>
__global__ void k_build_cells(const float* __restrict__ vol, int n, CellT<T>* __restrict__ cells) {
  const long nc = n + 1;
  const long total = nc * nc * nc;
  for (long ci = blockIdx.x * (long)blockDim.x + threadIdx.x; ci < total; ci += (long)gridDim.x * blockDim.x) {
    const int i = (int)(ci % nc) - 1, j = (int)((ci / nc) % nc) - 1, k = (int)(ci / (nc * nc)) - 1;
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int x = i + (q & 1), y = j + ((q >> 1) & 1), z = k + ((q >> 2) & 1);
      v[q] = (x >= 0 && y >= 0 && z >= 0 && x < n && y < n && z < n) ? vol[((long)z * n + y) * n + x] : 0.f;
    }
    CellT<T> c;
    if constexpr (sizeof(T) == 4) {
      reinterpret_cast<CellT<float>&>(c).lo = make_float4(v[0], v[1], v[2], v[3]);
      reinterpret_cast<CellT<float>&>(c).hi = make_float4(v[4], v[5], v[6], v[7]);
    } else {
      __nv_bfloat162* p = reinterpret_cast<__nv_bfloat162*>(&reinterpret_cast<CellT<__nv_bfloat16>&>(c).v);
#pragma unroll
      for (int q = 0; q < 4; ++q) p[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
    }
    cells[ci] = c;
  }
}

struct EvalItem {
  int particle;
  int orient;          // global orientation index
};

struct EvalStats {
  double sum_r, sum_r2, energy_spec, pad;
};

// Result of one evaluation: normalised CC at the peak and the integer shift.
struct EvalResult {
  float cc;
  int peak[3];
};

struct SearchChunkArgs {
  const EvalItem* items;     // [E]
  const DevParticle* parts;
  const DevRef* refs;
  const double* dmat;        // [norient][9] column-major defineMatrix([phi,theta,psi-phi],'inv')
  float2* s1;                // [E][ky][part][lpos(z)][TPB_K] slabs, S1_EVAL per evaluation
  float2* s2;                // [E][w][lpos(ky)][PC] planes, S2_PLANE each
  EvalStats* stats;          // [E]
  unsigned long long* keys;  // [E]
  int n_items;
  int radius;
  int interp;
  // With `done` set, the last pass-C CTA of an evaluation decodes it into results / best_keys
  // and clears its stats, key and counter for the next chunk.
  unsigned* done = nullptr;                  // [E] pass-C CTAs finished
  EvalResult* results = nullptr;             // [total evaluations of the run]
  unsigned long long* best_keys = nullptr;   // [particles]
  // Bounded device-side waits: a wait that gives up after wait_cycles SM clock cycles ORs
  // kStatusWaitTimeout into *status (when set) and its CTA returns without a result.
  unsigned* status = nullptr;
  long long wait_cycles = 1ll << 31;         // about a second at the B200's 1.965 GHz
  unsigned phantom_tx = 0;                   // test hook: bytes announced but never copied (0)
};
constexpr unsigned kStatusWaitTimeout = 1u;

// Decodes evaluation e of a chunk from its peak key and folds it into its particle's
// best-orientation key (cc, then the first orientation on ties).
__device__ __forceinline__ void decode_eval(const SearchChunkArgs& a, int n, int e, unsigned long long key) {
  const EvalItem it = a.items[e];
  const DevParticle& pt = a.parts[it.particle];
  EvalResult r;
  const int c = n / 2;
  if (key == 0ull) {
    r.cc = __int_as_float(0x7fc00000);
    r.peak[0] = r.peak[1] = r.peak[2] = 0;
  } else {
    r.cc = key_to_float((unsigned int)(key >> 32));
    const unsigned int lin = 0xffffffffu - (unsigned int)(key & 0xffffffffull);
    r.peak[0] = (int)(lin % n) - c;
    r.peak[1] = (int)((lin / n) % n) - c;
    r.peak[2] = (int)(lin / ((unsigned)n * n)) - c;
  }
  a.results[pt.eval_base + (it.orient - pt.orient_begin)] = r;
  if (key != 0ull) {
    const unsigned long long bk = ((unsigned long long)ordered_key(r.cc) << 32) | (0xffffffffu - (unsigned)it.orient);
    atomicMax(a.best_keys + it.particle, bk);
  }
}

// Sampling matrix rows of RotMat' with RotMat = prior * D (FP64 composition).
__device__ __forceinline__ void compose_sampling_matrix(const double* prior, const double* d, float m[9]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      // RotMat(j, i) = sum_k prior(j, k) D(k, i)
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < 3; ++k) acc = fma(prior[j + 3 * k], d[k + 3 * i], acc);
      m[3 * i + j] = (float)acc;
    }
}

// Default planes per pass-A CTA; the autotuner of search.cu may pick another supported value.
__host__ __device__ constexpr int default_planes(int N) { return N <= 64 ? 4 : (N <= 96 ? 2 : 1); }

template <int N, int GG = 0>
struct SearchCfg {
  static constexpr int NH = N / 2 + 1;
  static constexpr int P = team_size(N);
  static constexpr int G = GG ? GG : default_planes(N);  // planes per pass-A CTA
  static constexpr int NT_A = 256;
  static constexpr int TEAMS_A = NT_A / P;
  // Pass C uses half as many teams as the y transforms have lines (two rounds of y lines), so
  // that the C2R phase, where (2 r + 1 + 1) / 2 row pairs (8 at r = 7) keep as many teams busy,
  // leaves fewer idle and more CTAs fit per SM: 64^3 20 teams of 8 lanes, six CTAs per SM at 64
  // registers (88.7 us per 602-evaluation chunk against 131.1 with 33 teams); 96^3 28 teams and
  // 128^3 36, where the whole-row CTAs (416 and 544 threads) fitted once per SM by registers
  static constexpr int NT_BC = ((NH * P / 2 + 31) / 32) * 32;
  static constexpr int MINB_C = N <= 64 ? 6 : 2;
  static constexpr int TEAMS_BC = NT_BC / P;
  // FFT lines use padded positions (lpos<1>): a strided line of N elements spans PY rows, a
  // contiguous line buffer LP slots; LP = 8 (mod 16) puts neighbouring teams 16 banks apart.
  static constexpr int PY = padded_len(N);
  static constexpr int LP = PY + ((8 - PY % 16) + 16) % 16;
  // teams with a line buffer for the row-pair transforms (pass A R2C, pass C C2R); the others
  // idle during those loops, which keeps two pass-A CTAs per SM for every box size
  static constexpr int TEAMS_LA = N <= 64 ? TEAMS_A : 16;
  static constexpr int TEAMS_LC = 16;  // (2 r + 1 + 1) / 2 <= 16 row pairs for r <= 15
  static_assert(TEAMS_BC >= TEAMS_LC, "pass C needs a team for every line buffer");
  // Plane pitch of pass A (float2): nh rounded up to even.  With the even pitch the y transform's
  // teams take consecutive columns, the row-pair R2C's four teams of a warp take the pairs
  // q, q+2, q+1, q+3 of a group of four, and a bank model of every access puts each half-warp's
  // two teams on complementary banks in the R2C's reads and writes and in every y-transform stage
  // (64^3: 512 -> 256 R2C wavefronts per CTA; 96^3 / 128^3 also 3456 -> 2016 / 4096 -> 2560 in the
  // y transform); the slab store then reads column pairs as 16-byte words.
  static constexpr int PA = NH + (NH & 1);
  static constexpr size_t SMEM_A = sizeof(float2) * ((size_t)G * PY * PA + (size_t)TEAMS_LA * LP + N) + 64;
  // resident pass-A CTAs per SM that shared memory allows (228 KB per SM, 1 KB reserved per CTA),
  // and the target the register budget is capped for: 5 at 64^3 with one plane per CTA (48
  // registers, a 12-byte spill; 863.7 us per 602-evaluation chunk against 875.2 at the compiler's
  // 64 registers and 4 CTAs), none for the multi-plane 64^3 tilings, 2 for the larger boxes, whose
  // FFT codelets need more registers
  static constexpr int SMEM_CTAS_A = (int)((228 * 1024) / (SMEM_A + 1024));
  static constexpr int MINB_A = N <= 64 ? (G == 1 ? 5 : 0) : (SMEM_CTAS_A < 2 ? SMEM_CTAS_A : 2);
  // Pass B: a CTA transforms the z lines of one ky and one of KS_B parts of the kx columns (NHB
  // columns at most).  128^3 splits the columns in two: with the whole ky row a CTA needed 544
  // threads and 95 registers (one CTA per SM, latency-bound); half rows fit three per SM.  At 96^3
  // two parts (four CTAs per SM instead of two) took pass B from 494 to 448 us per chunk, but pass A's
  // stores of the second part, which starts at an odd column, from 965 to 1035 us.
  // Pass A writes S1 as pass B's shared-memory tiles: per (evaluation, ky, column part) a slab of PY
  // rows (row z at lpos<1>(z)) of TPB_K float2, which pass B fetches with one bulk copy.  The
  // particle spectrum and weight rows (the caller's layout) come in 16-byte cp.async pieces from the
  // 16-byte boundary at or below each row start, into rows of even pitch (QP_K float2, WP_K floats),
  // and are read at the row's offset from that boundary (the same for every row of a CTA: a z step
  // is N NH elements, a multiple of 16 bytes).  The teams of a warp take consecutive columns: with
  // the even tile pitch the two teams of a half-warp fall on complementary banks in every stage at
  // 64^3 (96^3 and 128^3 keep the few conflicts their radix-3 / radix-16 stages had with an odd
  // pitch), and the four of a warp read the weight rows (pitch WP_K) on disjoint banks.
  static constexpr int KS_B = N >= 128 ? 2 : 1;
  static constexpr int NHB = (NH + KS_B - 1) / KS_B;
  static constexpr int NT_B = ((NHB * P + 31) / 32) * 32;
  static constexpr int TEAMS_B = NT_B / P;
  static constexpr int GRID_BX = N * KS_B;
  // evaluations per pass-B CTA (grid y = ceil(items / EVALS_B)): four at 64^3 and 96^3, two at
  // 128^3, where the later ones reuse the particle's spectrum (and weight) rows (64^3: pass B 321.5 ->
  // 309.9 us per 534-evaluation chunk with two, 302.1 with four; 96^3, 69 registers, still two CTAs
  // per SM: 493.4 -> 505.6 us per 167-evaluation chunk with two, 485.3 with four; 128^3, 56
  // registers, three CTAs per SM: 446.4 -> 432.6 us per 72-evaluation chunk with two, 436.6 with
  // four).  A second slab tile, the next evaluation's slab copied while the current one is
  // transformed (66 KB, three CTAs per SM), took pass B from 295.6 to 307.0 us and the overlapped
  // 64^3 run from 620 to 679 ms: pass A of the other chunk no longer fits beside three such CTAs.
  static constexpr int EVALS_B = N <= 96 ? 4 : 2;
  static constexpr int TPB_K = NHB + 1 + (NHB + 1) % 2;                 // >= NHB + 1, even
  static constexpr int QP_K = TPB_K;
  static constexpr int WP_K = ((NHB + 3 + 3) / 4) * 4;                   // >= NHB + 3, 16-byte rows
  // The weight rows are copied too up to 96^3; at 128^3 the weight is read from L2 when the product
  // is formed, so that three CTAs per SM fit in shared memory instead of two.
  static constexpr bool PREF_W = N <= 96;
  // S1 elements per evaluation: a slab per (ky, column part)
  static constexpr size_t S1_EVAL = (size_t)N * KS_B * PY * TPB_K;
  static constexpr size_t SMEM_B = sizeof(float2) * ((size_t)PY * TPB_K + (size_t)N * QP_K + N) +
                                   (PREF_W ? sizeof(float) * (size_t)N * WP_K : 0);
  // Pass C's tile: S2 planes are written by pass B in this layout (rows ky at lpos<1>(ky), even
  // pitch PC), so pass C brings a plane in with one bulk copy; its y transforms then take
  // consecutive columns (a bank model gives the same wavefronts as the odd pitch with paired
  // columns).
  static constexpr int PC = NH + (NH & 1);
  static constexpr size_t S2_PLANE = (size_t)PY * PC;
  static constexpr size_t SMEM_C = sizeof(float2) * (S2_PLANE + N + (size_t)TEAMS_LC * LP);
};

// S1 elements per evaluation of box n (slabs padded to the z pass's tiles).
inline size_t s1_eval_elems(int n) {
  return n == 64 ? SearchCfg<64>::S1_EVAL : n == 96 ? SearchCfg<96>::S1_EVAL : SearchCfg<128>::S1_EVAL;
}
// S2 elements per output plane of box n (pass C's tile layout).
inline size_t s2_plane_elems(int n) {
  return n == 64 ? SearchCfg<64>::S2_PLANE : n == 96 ? SearchCfg<96>::S2_PLANE : SearchCfg<128>::S2_PLANE;
}

template <typename Tv>
__device__ __forceinline__ Tv block_sum(Tv v, Tv* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  Tv t = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
  return t;  // valid in thread 0
}

// Gather of the G planes of pass A through corner cells.  Each warp takes RU whole rows per step;
// lane l samples x = l + 32 k (k < N / 32) of each, so one load instruction of a warp covers 32
// consecutive voxels of a row (neighbouring cells, few L1 lines per request).  A thread computes
// its sample point once per row and steps 32 voxels along x by adding 32 x (first column of the
// sampling matrix); its RU * N / 32 cell loads are all issued before any is used.  Sums of r and
// r^2 are formed per step in FP32 and accumulated in FP64.
// A lane whose voxel lies outside its row's mask extent (mask_rows) skips its cell: it reads cell 0,
// which every such lane of the warp shares, and its value is 0 as the mask would make it.
template <int N, typename T, int MODE, int GG>
__device__ __forceinline__ void gather_cells(const CellT<T>* __restrict__ cells, const float* __restrict__ mask,
                                             const unsigned* __restrict__ mask_rows, const float m[9], float tx,
                                             float ty, float tz, int z0, float* __restrict__ fplanes, double& s1,
                                             double& s2) {
  using C = SearchCfg<N, GG>;
  constexpr int G = C::G, NT = C::NT_A;
  constexpr int SEG = N / 32;                     // row segments per lane
  constexpr int RU = SEG >= 3 ? 2 : 4 / SEG;      // rows per warp per step: U = RU * SEG loads in flight
  // (two rows at 96^3 / 128^3: 6 / 8 cells in flight; 128^3 pass A 149 us per 9 evaluations from 156)
  constexpr int U = RU * SEG;
  constexpr int WARPS = NT / 32;
  constexpr int ROWS = G * N;
  static_assert(N % 32 == 0 && ROWS % (WARPS * RU) == 0, "gather tiling");
  constexpr int c = N / 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float step_x = 32.f * m[0], step_y = 32.f * m[3], step_z = 32.f * m[6];
#pragma unroll 1
  for (int r0 = warp * RU; r0 < ROWS; r0 += WARPS * RU) {
    CellT<T> cv[U];
    float fr[U][3];
    bool ok[U];
    float mk[U];
#pragma unroll
    for (int ru = 0; ru < RU; ++ru) {
      const int row = r0 + ru, y = row % N, zl = row / N, z = z0 + zl;
      const unsigned ext = mask_rows ? __ldg(mask_rows + z * N + y) : ((unsigned)N << 16);
      const int lo = (int)(ext & 0xffffu), hi = (int)(ext >> 16);
      const float pu = (float)(lane - c) - tx, pv = (float)(y - c) - ty, pw = (float)(z - c) - tz;
      float sx = fmaf(m[0], pu, fmaf(m[1], pv, m[2] * pw)) + (float)c;
      float sy = fmaf(m[3], pu, fmaf(m[4], pv, m[5] * pw)) + (float)c;
      float sz = fmaf(m[6], pu, fmaf(m[7], pv, m[8] * pw)) + (float)c;
#pragma unroll
      for (int k = 0; k < SEG; ++k) {
        const int u = ru * SEG + k;
        const int x = lane + 32 * k;
        const bool in = x >= lo && x < hi;
        unsigned ci = cell_index_gather<MODE>(N, sx, sy, sz, fr[u], ok[u]);
        ci = in ? ci : 0u;
        ok[u] = ok[u] && in;
        cv[u] = load_cell(cells + ci);
        mk[u] = !mask ? 1.f : (in ? __ldg(mask + ((long)z * N + y) * N + x) : 0.f);
        sx += step_x;
        sy += step_y;
        sz += step_z;
      }
    }
    float p1 = 0.f, p2 = 0.f;
#pragma unroll
    for (int ru = 0; ru < RU; ++ru) {
      const int row = r0 + ru, y = row % N, zl = row / N;
      float* dst = fplanes + ((size_t)zl * C::PY + lpos<1>(y)) * (2 * C::PA) + lane;
#pragma unroll
      for (int k = 0; k < SEG; ++k) {
        const int u = ru * SEG + k;
        float cvv[8];
        cell_values(cv[u], cvv);
        const float val = (ok[u] ? cell_trilinear(cvv, fr[u]) : 0.f) * mk[u];
        dst[32 * k] = val;
        p1 += val;
        p2 = fmaf(val, val, p2);
      }
    }
    s1 += (double)p1;
    s2 += (double)p2;
  }
}

// ------------------------------------------------------------------ pass A
template <int N, typename T, int GG = 0>
__global__ void __launch_bounds__(SearchCfg<N, GG>::NT_A, SearchCfg<N, GG>::MINB_A) k_search_fwd_xy(const SearchChunkArgs a,
                                                                           const float2* __restrict__ g_tw) {
  using C = SearchCfg<N, GG>;
  constexpr int NH = C::NH, G = C::G, P = C::P;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PY = C::PY, LP = C::LP;
  constexpr int PA = C::PA;
  float2* planes = reinterpret_cast<float2*>(smem_raw);          // [G][PY][PA], row y at lpos<1>(y)
  float2* lines = planes + (size_t)G * PY * PA;                   // [TEAMS][LP]
  float2* s_tw = lines + (size_t)C::TEAMS_LA * LP;                 // [N]
  float* s_m = reinterpret_cast<float*>(s_tw + N);                // 9 floats
  __shared__ double red[2][32];

  const int e = blockIdx.y;
  if (e >= a.n_items) return;
  const int z0 = blockIdx.x * G;
  const EvalItem it = a.items[e];
  const DevParticle& pt = a.parts[it.particle];
  const DevRef rf = a.refs[pt.ref];
  const T* __restrict__ src = reinterpret_cast<const T*>(rf.data);
  const float* __restrict__ mask = rf.mask;

  load_twiddles<N>(s_tw, g_tw);
  if (threadIdx.x == 0) compose_sampling_matrix(pt.prior, a.dmat + 9L * it.orient, s_m);
  __syncthreads();
  float m[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) m[i] = s_m[i];
  const float tx = pt.shift[0], ty = pt.shift[1], tz = pt.shift[2];
  constexpr int c = N / 2;

  // 1. gather (x fastest: a warp walks 32 consecutive voxels of one row)
  double s1 = 0.0, s2 = 0.0;
  float* fplanes = reinterpret_cast<float*>(planes);
  if (rf.cells && a.interp == EMC_INTERP_LINEAR) {
    gather_cells<N, T, EMC_INTERP_LINEAR, GG>(reinterpret_cast<const CellT<T>*>(rf.cells), mask, rf.mask_rows, m, tx,
                                              ty, tz, z0, fplanes, s1, s2);
  } else if (rf.cells && a.interp == EMC_INTERP_LINEAR_BORDER) {
    gather_cells<N, T, EMC_INTERP_LINEAR_BORDER, GG>(reinterpret_cast<const CellT<T>*>(rf.cells), mask, rf.mask_rows,
                                                     m, tx, ty, tz, z0, fplanes, s1, s2);
  } else {
    for (int idx = threadIdx.x; idx < G * N * N; idx += C::NT_A) {
      const int x = idx % N, y = (idx / N) % N, zl = idx / (N * N);
      const int z = z0 + zl;
      const float u = (float)(x - c) - tx, v = (float)(y - c) - ty, w = (float)(z - c) - tz;
      const float sx = fmaf(m[0], u, fmaf(m[1], v, m[2] * w)) + (float)c;
      const float sy = fmaf(m[3], u, fmaf(m[4], v, m[5] * w)) + (float)c;
      const float sz = fmaf(m[6], u, fmaf(m[7], v, m[8] * w)) + (float)c;
      float val = sample(a.interp, src, N, N, N, sx, sy, sz);
      if (mask) val *= __ldg(mask + ((long)z * N + y) * N + x);
      fplanes[((size_t)zl * PY + lpos<1>(y)) * (2 * PA) + x] = val;
      s1 += (double)val;
      s2 += (double)val * (double)val;
    }
  }
  if (!(rf.wref || pt.wedge)) {
    // E_R from the real-space sums (Parseval) is needed only without a weight on the reference;
    // with one, pass B forms the weighted spectral energy (the branch is uniform over the block)
    double t1 = block_sum(s1, red[0]);
    double t2 = block_sum(s2, red[1]);
    if (threadIdx.x == 0) {
      atomicAdd(&a.stats[e].sum_r, t1);
      atomicAdd(&a.stats[e].sum_r2, t2);
    }
  }
  __syncthreads();

  const int team = threadIdx.x / P, lane = threadIdx.x % P;
  LineTw<N, P> tc;
  tc.init(s_tw, lane);
  // 2. R2C along x: rows 2q and 2q+1 of the slab share one complex FFT
  {
    constexpr int NPAIRS = G * N / 2;
    const bool has_line = team < C::TEAMS_LA;
    float2* buf = lines + (size_t)(has_line ? team : 0) * LP;
    static_assert((C::TEAMS_LA * P) % 32 == 0, "line-buffer teams fill whole warps");
    // warps without line buffers (96^3, 128^3: the second half of the CTA) skip the loop
    for (int base = 0; base < NPAIRS && threadIdx.x < C::TEAMS_LA * P; base += C::TEAMS_LA) {
      const int q = base + ((team & ~3) | ((team & 1) << 1) | ((team >> 1) & 1));  // pairs 0, 2, 1, 3
      const bool active = has_line && q < NPAIRS;
      // rows 2q, 2q+1 of the slab (same plane, adjacent padded rows since 2q+1 is odd)
      const int zl = (2 * q) / N, ya = (2 * q) % N;
      const size_t row_a = (size_t)zl * PY + lpos<1>(ya);
      const float* ra = fplanes + row_a * (2 * PA);
      const float* rb = ra + 2 * PA;
      // the transform's last stage stays in registers: v[b][r] = Z(k), k = lane + b P + NSL r
      using LS = LastStage<N, P>;
      float2 v[LS::PER][LS::RL];
      fft_line_in_regs<N, -1, P, 1>([&](int n) { return make_float2(ra[n], rb[n]); }, buf, 1, lane, s_tw, active,
                                    &tc, v);
      // Hermitian split of the two packed rows: Z(N - k) sits on lane (P - lane) mod P of the team,
      // butterfly block NSL/P - 1 - b, index RL - 1 - r (lane 0 holds its own partners and Z(N/2)).
      // Columns 0 and N/2 of a row transform are real: row a's pair goes to slot 0 of row a, row
      // b's to slot 0 of row b, as (X(0), X(N/2)), so the y pass needs N/2 complex lines.
      constexpr int NB_P = LS::NSL / P;
      constexpr int JH = (N / 2) % LS::NSL, BH = JH / P, RH = (N / 2) / LS::NSL;
      static_assert(JH % P == 0 && LS::NSL % P == 0, "Z(N/2) on lane 0");
      const int wl = threadIdx.x & 31;
      const int src = (wl & ~(P - 1)) | ((P - lane) & (P - 1));
      float2* oa = planes + row_a * PA;
      float2* ob = oa + PA;
#pragma unroll
      for (int b = 0; b < LS::PER; ++b) {
#pragma unroll
        for (int r = 0; r < LS::RL; ++r) {
          if (b * P + r * LS::NSL < N / 2) {
            const float2 sent = v[NB_P - 1 - b][LS::RL - 1 - r];
            float2 zm = make_float2(__shfl_sync(0xffffffffu, sent.x, src), __shfl_sync(0xffffffffu, sent.y, src));
            if (lane == 0) {
              zm = b > 0 ? v[(NB_P - b) % LS::PER][LS::RL - 1 - r] : (r > 0 ? v[0][(LS::RL - r) % LS::RL] : v[BH][RH]);
            }
            const float2 zk = v[b][r];
            const int k = lane + b * P + r * LS::NSL;
            if (active && k < N / 2) {
              if (k == 0) {
                oa[0] = make_float2(zk.x, zm.x);
                ob[0] = make_float2(zk.y, zm.y);
              } else {
                oa[k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
                ob[k] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
              }
            }
          }
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();
  // 3. FFT along y for columns 0 .. N/2-1 of every plane (column 0 carries X(0) + i X(N/2))
  {
    constexpr int NLINES = G * (N / 2);
    static_assert(NLINES % (32 / P) == 0, "a warp's teams are all active or all idle");
    for (int base = 0; base < NLINES; base += C::TEAMS_A) {
      // a warp whose teams all lie past the last line (96^3: the second round) skips the round
      if (base + (int)(threadIdx.x >> 5) * (32 / P) >= NLINES) continue;
      const int li = base + team;
      const bool active = li < NLINES;
      const int zl = active ? li / (N / 2) : 0, kx = active ? li % (N / 2) : 0;
      fft_line<N, -1, P, 1>(planes + (size_t)zl * PY * PA + kx, PA, lane, s_tw, active, &tc);
    }
  }
  __syncthreads();
  // 4. store plane z0 + zl into the S1 slabs (row lpos(z) of slab (ky = y, column part)), values
  //    gathered from their padded positions; columns 0 and N/2 are separated from the packed
  //    column 0: with Z = F(X(0) + i X(N/2)),
  //    F X(0)(y) = (Z(y) + conj Z(-y)) / 2 and F X(N/2)(y) = (Z(y) - conj Z(-y)) / 2i
  {
    // F X(kx)(y) of local plane zl: columns 0 and N/2 separated from the packed column 0
    auto s1_value = [&](int zl, int y, int kx) {
      const float2* pl = planes + (size_t)zl * PY * PA;
      if (kx >= NH) return make_float2(0.f, 0.f);
      if (kx == 0 || kx == NH - 1) {
        const float2 zp = pl[lpos<1>(y) * PA], zm = pl[lpos<1>((N - y) % N) * PA];
        return kx == 0 ? make_float2(0.5f * (zp.x + zm.x), 0.5f * (zp.y - zm.y))
                       : make_float2(0.5f * (zp.y + zm.y), -0.5f * (zp.x - zm.x));
      }
      return pl[lpos<1>(y) * PA + kx];
    };
    float2* dst = a.s1 + (size_t)e * C::S1_EVAL;
    {
      // slabs [ky][part][lpos(z)][TPB_K] (part: columns [part NHB, part NHB + NHB)): whole rows, pad
      // columns zero, two elements per 16-byte store
      constexpr int RP = C::TPB_K / 2, KS = C::KS_B, NB = C::NHB;
      constexpr int NV = G * N * KS * RP;
      for (int i = threadIdx.x; i < NV; i += C::NT_A) {
        const int row = i / (KS * RP), rem = i % (KS * RP);  // row = zl * N + y
        const int part = rem / RP, c = rem % RP;
        const int zl = row / N, y = row % N;
        const int k0 = part * NB + 2 * c;
        float2 v0, v1;
        if (k0 % 2 == 0 && k0 + 1 < NH - 1 && k0 != 0 && 2 * c + 1 < NB) {
          // an ordinary column pair: one 16-byte read (even pitch, even column)
          const float4 q4 = *reinterpret_cast<const float4*>(planes + ((size_t)zl * PY + lpos<1>(y)) * PA + k0);
          v0 = make_float2(q4.x, q4.y);
          v1 = make_float2(q4.z, q4.w);
        } else {
          v0 = 2 * c < NB ? s1_value(zl, y, k0) : make_float2(0.f, 0.f);
          v1 = 2 * c + 1 < NB ? s1_value(zl, y, k0 + 1) : make_float2(0.f, 0.f);
        }
        *reinterpret_cast<float4*>(dst + (((size_t)y * KS + part) * PY + lpos<1>(z0 + zl)) * C::TPB_K + 2 * c) =
            make_float4(v0.x, v0.y, v1.x, v1.y);
      }
    }
  }
}

// ------------------------------------------------------------------ pass B
// Pass B: pass A left the (evaluation, ky, column part) slab in the tile's
// layout, so one cp.async.bulk completed on an mbarrier brings it in; the particle spectrum and
// weight rows arrive meanwhile as 16-byte cp.async pieces, and the fused z lines read them at the
// rows' offsets from their 16-byte boundaries.  A spectrum or weight whose base is not 16-byte
// aligned (a caller's buffer at an odd element offset) is copied element by element, at offset 0.
template <int N>
__device__ __forceinline__ void z_mul_bulk(const SearchChunkArgs& a, const float2* __restrict__ g_tw) {
  using C = SearchCfg<N>;
  constexpr int NH = C::NH, P = C::P, NT = C::NT_B, NB = C::NHB, TP = C::TPB_K, QP = C::QP_K, WP = C::WP_K;
  static_assert(C::TEAMS_B >= NB, "one round of z lines");
  constexpr unsigned SLAB_BYTES = (unsigned)(sizeof(float2) * C::PY * TP);
  static_assert(SLAB_BYTES % 16 == 0, "bulk copy size");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tile = reinterpret_cast<float2*>(smem_raw);                // [PY][TP], row z at lpos<1>(z)
  float2* s_q = tile + (size_t)C::PY * TP;                            // [N][QP]
  float* s_w = reinterpret_cast<float*>(s_q + (size_t)N * QP);       // [N][WP] (PREF_W)
  float2* s_tw = reinterpret_cast<float2*>(s_w + (C::PREF_W ? (size_t)N * WP : 0));  // [N]
  __shared__ double red[32];
  __shared__ uint64_t bar;

  // EVALS_B consecutive evaluations of the chunk (consecutive orientations of one particle, but at
  // a particle boundary): the spectrum and weight rows are copied again only when the particle changes
  const int e_first = blockIdx.y * C::EVALS_B;
  if (e_first >= a.n_items) return;
  const int ne = min(C::EVALS_B, a.n_items - e_first);
  // this CTA's columns: kx in [k0, k0 + cnt)
  const int ky = blockIdx.x / C::KS_B;
  const int k0 = (int)(blockIdx.x % C::KS_B) * NB;
  const int cnt = min(NB, NH - k0);
  const int w = 2 * a.radius + 1;
  constexpr size_t ZS = (size_t)N * NH;  // elements per z step of the spectrum and weight
  const int team = threadIdx.x / P, lane = threadIdx.x % P;
  const int kl = team;  // consecutive columns for the teams of a warp
  const int kx = k0 + kl;
  const double hw = (kx == 0 || 2 * kx == N) ? 1.0 : 2.0;

  if (threadIdx.x == 0) mbar_init(&bar, 1);
  load_twiddles<N>(s_tw, g_tw);
  __syncthreads();  // the barrier is initialised before anyone polls it
  int loaded = -1;  // particle whose spectrum and weight rows are in shared memory
  // one evaluation; returns false when its copy timed out (the CTA then leaves)
  auto one = [&](const int k) -> bool {
    const int e = e_first + k;
    const EvalItem it = a.items[e];
    const DevParticle& pt = a.parts[it.particle];
    // weights on the rotated reference (BH_multi_xcf_Translational_2.m:35-38): the particle's
    // wdgMask and the reference's bandpass wref; the first present one is copied, a second folded in
    const float* __restrict__ wref = a.refs[pt.ref].wref;
    const float* __restrict__ w1 = pt.wedge ? pt.wedge : wref;
    const float* __restrict__ w2 = pt.wedge ? wref : nullptr;
    const float2* qrow = pt.spec + (size_t)ky * NH + k0;
    const float* wrow = w1 ? w1 + (size_t)ky * NH + k0 : nullptr;
    const bool piece_q = ((uintptr_t)pt.spec & 15) == 0;
    const bool piece_w = C::PREF_W && w1 && ((uintptr_t)w1 & 15) == 0;
    // row offsets (elements) from the 16-byte boundary below each row start, 16-byte pieces per row
    const int offq = piece_q ? (int)(((uintptr_t)qrow & 15) >> 3) : 0;
    const int offw = piece_w ? (int)(((uintptr_t)wrow & 15) >> 2) : 0;
    const bool reload = it.particle != loaded;  // the same for the whole CTA
    if (k > 0) __syncthreads();  // the previous evaluation is done with the tile (and the rows)
    if (threadIdx.x == 0) {
      if (k > 0) fence_proxy_async_shared();
      mbar_arrive_expect_tx(&bar, SLAB_BYTES + a.phantom_tx);
      bulk_copy_g2s(tile, a.s1 + (size_t)e * C::S1_EVAL + (size_t)blockIdx.x * C::PY * TP, SLAB_BYTES, &bar);
    }
    if (reload) {
      const int pq = ((offq + cnt) * 8 + 15) >> 4;
      const int pw = ((offw + cnt) * 4 + 15) >> 4;
      if (piece_q) {
        const char* src = reinterpret_cast<const char*>(qrow - offq);
        for (int i = threadIdx.x; i < N * pq; i += NT) {
          const int z = i / pq, c = i % pq;
          cp_async16(reinterpret_cast<char*>(s_q + (size_t)z * QP) + 16 * c, src + z * ZS * sizeof(float2) + 16 * c);
        }
      } else {
        for (int i = threadIdx.x; i < N * NB; i += NT)
          if (i % NB < cnt) cp_async8(s_q + (i / NB) * QP + i % NB, qrow + (i / NB) * ZS + i % NB);
      }
      if (piece_w) {
        const char* src = reinterpret_cast<const char*>(wrow - offw);
        for (int i = threadIdx.x; i < N * pw; i += NT) {
          const int z = i / pw, c = i % pw;
          cp_async16(reinterpret_cast<char*>(s_w + (size_t)z * WP) + 16 * c, src + z * ZS * sizeof(float) + 16 * c);
        }
      } else if (C::PREF_W && w1) {
        for (int i = threadIdx.x; i < N * NB; i += NT)
          if (i % NB < cnt) cp_async4(s_w + (i / NB) * WP + i % NB, wrow + (i / NB) * ZS + i % NB);
      }
      cp_async_commit();
      cp_async_wait<0>();
    }
    // the next barrier also publishes the cp.async pieces; the whole CTA takes the same branch
    const bool arrived = mbar_wait(&bar, (unsigned)(k & 1), a.wait_cycles);
    if (__syncthreads_or(!arrived)) {
      // the copy did not complete in time: report, give it a second bounded wait, and leave
      if (threadIdx.x == 0 && a.status) atomicOr(a.status, kStatusWaitTimeout);
      mbar_wait(&bar, (unsigned)(k & 1), a.wait_cycles);
      return false;
    }
    if (reload) {
      if (C::PREF_W && w2) {
        for (int i = threadIdx.x; i < N * NB; i += NT)
          if (i % NB < cnt)
            s_w[(i / NB) * WP + offw + i % NB] *= __ldg(w2 + (size_t)(i / NB) * ZS + (size_t)ky * NH + k0 + i % NB);
        __syncthreads();
      }
      loaded = it.particle;
    }

    const bool weighted = w1 != nullptr;
    // E_R: each lane's |.|^2 over its elements of the line (8 to 16) in FP32, the lanes' partial
    // sums then accumulated in FP64 (block_sum and the evaluation's atomicAdd)
    float ef = 0.f;
    {
      const float2* sq = s_q + offq + kl;
      const float* sw = s_w + offw + kl;
      fft_line_fwd_mul_inv<N, P, 1>(tile + kl, TP, lane, s_tw, kl < cnt, [&](int z, float2 rr) {
        const bool origin = z == 0 && ky == 0 && kx == 0;
        if (weighted) {
          float wv;
          if constexpr (C::PREF_W) {
            wv = sw[z * WP];
          } else {  // read when the product is formed (128^3: no weight slab, three CTAs per SM)
            const size_t gi = (size_t)z * ZS + (size_t)ky * NH + kx;
            wv = __ldg(w1 + gi);
            if (w2) wv *= __ldg(w2 + gi);
          }
          rr.x *= wv;
          rr.y *= wv;
          if (!origin) ef = fmaf(rr.x, rr.x, fmaf(rr.y, rr.y, ef));
        }
        const float2 x = cmulc(sq[z * QP], rr);
        return origin ? make_float2(0.f, 0.f) : x;
      });
    }
    if (weighted) {
      double t = block_sum(hw * (double)ef, red);
      if (threadIdx.x == 0) atomicAdd(&a.stats[e].energy_spec, t);
    }
    __syncthreads();
    float2* dst = a.s2 + (size_t)e * w * C::S2_PLANE + (size_t)lpos<1>(ky) * C::PC + k0;
    for (int i = threadIdx.x; i < w * NB; i += NT) {
      const int j = i / NB, c = i % NB;
      if (c >= cnt) continue;
      const int z = (j - a.radius + N) % N;
      dst[(size_t)j * C::S2_PLANE + c] = tile[lpos<1>(z) * TP + c];
    }
    return true;
  };
  // straight-line calls (a rolled loop over evaluations let the compiler hoist the transforms'
  // addressing out of it and spill)
  static_assert(C::EVALS_B == 1 || C::EVALS_B == 2 || C::EVALS_B == 4, "1, 2 or 4 evaluations per CTA");
  if (!one(0)) return;
  if constexpr (C::EVALS_B > 1) {
    if (ne < 2 || !one(1)) return;
  }
  if constexpr (C::EVALS_B > 2) {
    if (ne < 3 || !one(2)) return;
    if (ne < 4) return;
    one(3);
  }
}

// 64^3: four resident 288-thread CTAs per SM asked of the compiler
template <int N>
__global__ void __launch_bounds__(SearchCfg<N>::NT_B, N <= 64 ? 4 : 0) k_search_z_mul(const SearchChunkArgs a,
                                                                      const float2* __restrict__ g_tw) {
  z_mul_bulk<N>(a, g_tw);
}

// ------------------------------------------------------------------ pass C
template <int N>
__global__ void __launch_bounds__(SearchCfg<N>::NT_BC, SearchCfg<N>::MINB_C) k_search_inv_peak(const SearchChunkArgs a,
                                                                          const float2* __restrict__ g_tw) {
  using C = SearchCfg<N>;
  constexpr int NH = C::NH, P = C::P;
  constexpr int PC = C::PC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tile = reinterpret_cast<float2*>(smem_raw);   // [PY][PC], row y at lpos<1>(y)
  float2* s_tw = tile + C::S2_PLANE;
  float2* lines = s_tw + N;                              // [TEAMS][LP]
  __shared__ unsigned long long s_best;
  __shared__ uint64_t bar;
  constexpr unsigned PLANE_BYTES = (unsigned)(sizeof(float2) * C::S2_PLANE);
  static_assert(PLANE_BYTES % 16 == 0, "bulk copy size");

  const int e = blockIdx.y;
  if (e >= a.n_items) return;
  const int j = blockIdx.x;
  const int r = a.radius, w = 2 * r + 1;
  const int sz = j - r;
  const EvalItem it = a.items[e];
  const DevParticle& pt = a.parts[it.particle];
  // with a weight on the reference E_R is its weighted spectral energy (pass B), else the
  // DC-free real-space energy of the rotated, masked reference (pass A, by Parseval)
  const bool weighted = a.refs[pt.ref].wref != nullptr || pt.wedge != nullptr;

  // the plane (pass B wrote it in this tile's layout) with one bulk copy, on a bounded wait
  if (threadIdx.x == 0) {
    s_best = 0ull;
    mbar_init(&bar, 1);
    mbar_arrive_expect_tx(&bar, PLANE_BYTES + a.phantom_tx);
    bulk_copy_g2s(tile, a.s2 + ((size_t)e * w + j) * C::S2_PLANE, PLANE_BYTES, &bar);
  }
  load_twiddles<N>(s_tw, g_tw);
  __syncthreads();  // the barrier is initialised before anyone polls it
  const bool arrived = mbar_wait(&bar, 0, a.wait_cycles);
  if (__syncthreads_or(!arrived)) {
    // the copy did not complete in time: report, give it a second bounded wait, and leave
    if (threadIdx.x == 0 && a.status) atomicOr(a.status, kStatusWaitTimeout);
    mbar_wait(&bar, 0, a.wait_cycles);
    return;
  }
  const int team = threadIdx.x / P, lane = threadIdx.x % P;
  LineTw<N, P> tc;
  tc.init(s_tw, lane);
  for (int base = 0; base < NH; base += C::TEAMS_BC) {
    const int li = base + team;  // consecutive columns for the teams of a warp
    fft_line<N, 1, P, 1>(tile + (li < NH ? li : 0), PC, lane, s_tw, li < NH, &tc);
  }
  __syncthreads();

  const EvalStats st = a.stats[e];
  const double er = weighted ? st.energy_spec : ((double)N * N * N * st.sum_r2 - st.sum_r * st.sum_r);
  const double denom = er * pt.energy;
  const float inv_norm = denom > 0.0 ? (float)(1.0 / sqrt(denom)) : 0.f;
  constexpr int c = N / 2;

  unsigned long long best = 0ull;
  // (warps with no row pair run the C2R loop predicated off; letting them skip it measured slower:
  // 74.2 -> 76-78 us per 64^3 chunk, a 4-byte spill and the branch against idle issue slots)
  const int npairs = (w + 1) / 2;
  const bool has_line = team < C::TEAMS_LC;
  float2* buf = lines + (size_t)(has_line ? team : 0) * C::LP;
  for (int base = 0; base < npairs; base += C::TEAMS_LC) {
    const int pr = base + team;
    const bool active = has_line && pr < npairs;
    const int ja = 2 * pr, jb = 2 * pr + 1;
    const bool has_b = jb < w;
    const int ya = (ja - r + N) % N, yb = has_b ? (jb - r + N) % N : ya;
    const float2* ra = tile + (size_t)lpos<1>(ya) * PC;
    const float2* rb = tile + (size_t)lpos<1>(yb) * PC;
    // Hermitian extension of rows a and b packed as a + i b
    fft_line_in<N, 1, P, 1>(
        [&](int n) {
          const bool lower = n <= N / 2;
          const int k = lower ? n : N - n;
          float2 A = ra[k];
          float2 B = has_b ? rb[k] : make_float2(0.f, 0.f);
          if (k == 0 || 2 * k == N) { A.y = 0.f; B.y = 0.f; }
          if (!lower) { A.y = -A.y; B.y = -B.y; }
          return make_float2(A.x - B.y, A.y + B.x);
        },
        buf, 1, lane, s_tw, active, &tc);
    if (active) {
      for (int t = lane; t < 2 * w; t += P) {
        const int which = t / w;  // 0: row a, 1: row b
        if (which == 1 && !has_b) continue;
        const int sx = (t % w) - r;
        const int sy = (which ? jb : ja) - r;
        if (sx * sx + sy * sy + sz * sz > r * r) continue;
        const float2 zv = buf[lpos<1>((sx + N) % N)];
        const float v = (which ? zv.y : zv.x) * inv_norm;
        if (v != v) continue;  // NaN never wins (MATLAB max ignores NaN)
        const unsigned int lin = (unsigned int)(((sz + c) * N + (sy + c)) * N + (sx + c));
        const unsigned long long key = ((unsigned long long)ordered_key(v) << 32) | (0xffffffffu - lin);
        best = key > best ? key : best;
      }
    }
    __syncwarp();
  }
  // block max
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, o);
    best = other > best ? other : best;
  }
  if ((threadIdx.x & 31) == 0 && best) atomicMax(&s_best, best);
  __syncthreads();
  if (threadIdx.x == 0 && s_best) atomicMax(&a.keys[e], s_best);
  if (a.done && threadIdx.x == 0) {
    // the last CTA of this evaluation (every other one has published its maximum) decodes it
    __threadfence();
    if (atomicAdd(&a.done[e], 1u) == (unsigned)(w - 1)) {
      __threadfence();
      const unsigned long long key = atomicExch(&a.keys[e], 0ull);
      decode_eval(a, N, e, key);
      a.stats[e] = EvalStats{0.0, 0.0, 0.0, 0.0};
      a.done[e] = 0u;
    }
  }
}

}  // namespace emc
