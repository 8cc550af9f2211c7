// search.cu -- host orchestration of the fused orientation search (C-ABI emc_search_*),
// particle-spectrum preparation and the real-space particle template.
//
// A run evaluates every (particle, orientation) pair of the request.  Pairs are grouped by
// (box size, reference storage type) and cut into chunks whose on-chip-spilled scratch
// (S1 + S2) stays inside a budget sized to the L2 cache; each chunk is four launches
// (fwd_xy, z_mul, inv_peak, decode).  The whole launch sequence of a run is captured once
// in a CUDA graph; the graphs of the four most recent requests (particles, outputs, settings)
// are kept, each with its own particle table, and replayed when a request repeats.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "fft_passes.cuh"
#include "search_kernels.cuh"

namespace emc {

__global__ void k_search_best(const DevParticle* __restrict__ parts, int np, const EvalResult* __restrict__ results,
                              const unsigned long long* __restrict__ best_keys, emc_search_hit* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const unsigned long long k = best_keys[p];
  emc_search_hit h;
  if (k == 0ull) {
    h.cc = __int_as_float(0x7fc00000);
    h.orient = -1;
    h.peak[0] = h.peak[1] = h.peak[2] = 0;
  } else {
    const int o = (int)(0xffffffffu - (unsigned int)(k & 0xffffffffull));
    const EvalResult r = results[parts[p].eval_base + (o - parts[p].orient_begin)];
    h.cc = r.cc;
    h.orient = o;
    h.peak[0] = r.peak[0]; h.peak[1] = r.peak[1]; h.peak[2] = r.peak[2];
  }
  out[p] = h;
}

// x extent of the non-zero mask voxels of every (z, y) row (lo = n, hi = 0 for an empty row).
__global__ void k_mask_rows(const float* __restrict__ mask, int n, unsigned* __restrict__ rows) {
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n * n) return;
  const float* m = mask + (long)row * n;
  int lo = n, hi = 0;
  for (int x = lane; x < n; x += 32)
    if (m[x] != 0.f) {
      lo = min(lo, x);
      hi = max(hi, x + 1);
    }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if (lane == 0) rows[row] = (unsigned)lo | ((unsigned)hi << 16);
}

// Particle energies taken from device memory (written there by emc_particle_spectrum) when the run
// executes, for emc_search_run_energies.
__global__ void k_search_energies(DevParticle* __restrict__ parts, int np, const double* __restrict__ energy) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < np) parts[p].energy = energy[p];
}

__global__ void k_search_scatter(const EvalResult* __restrict__ results, long n, float* __restrict__ cc,
                                 int* __restrict__ peak) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const EvalResult r = results[i];
    if (cc) cc[i] = r.cc;
    if (peak) { peak[3 * i] = r.peak[0]; peak[3 * i + 1] = r.peak[1]; peak[3 * i + 2] = r.peak[2]; }
  }
}

// ------------------------------------------------------------------ per-size dispatch
// Pass A holds G z-planes per CTA: larger G amortises the per-CTA setup (sampling matrix,
// twiddles, reductions) over more planes, smaller G raises the number of resident CTAs. The
// best G depends on the box, the chunk size (wave quantisation over the SMs) and the
// reference storage type, so it is chosen by timing (tune_planes) rather than fixed.
constexpr size_t kMaxSmemPerCta = 227 * 1024;
constexpr int kPlaneOptions[] = {1, 2, 4, 8};

template <int N, int G>
constexpr bool planes_fit() {
  return N % G == 0 && SearchCfg<N, G>::SMEM_A <= kMaxSmemPerCta;
}

template <int N, typename T, int G>
static emc_status set_attr_fwd() {
  if constexpr (planes_fit<N, G>())
    EMC_CUDA(cudaFuncSetAttribute(k_search_fwd_xy<N, T, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)SearchCfg<N, G>::SMEM_A));
  return EMC_OK;
}

template <int N, typename T>
static emc_status set_attrs() {
  using C = SearchCfg<N>;
  EMC_TRY((set_attr_fwd<N, T, 1>()));
  EMC_TRY((set_attr_fwd<N, T, 2>()));
  EMC_TRY((set_attr_fwd<N, T, 4>()));
  EMC_TRY((set_attr_fwd<N, T, 8>()));
  EMC_CUDA(cudaFuncSetAttribute(k_search_z_mul<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM_B));
  EMC_CUDA(cudaFuncSetAttribute(k_search_inv_peak<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM_C));
  return EMC_OK;
}

template <int N, typename T, int G>
static bool launch_fwd_g(const SearchChunkArgs& a, const float2* tw, cudaStream_t st) {
  if constexpr (planes_fit<N, G>()) {
    using C = SearchCfg<N, G>;
    k_search_fwd_xy<N, T, G><<<dim3(N / G, a.n_items), C::NT_A, C::SMEM_A, st>>>(a, tw);
    return true;
  }
  return false;
}

template <int N, typename T>
static emc_status launch_fwd(int g, const SearchChunkArgs& a, const float2* tw, cudaStream_t st) {
  bool ok = false;
  switch (g) {
    case 1: ok = launch_fwd_g<N, T, 1>(a, tw, st); break;
    case 2: ok = launch_fwd_g<N, T, 2>(a, tw, st); break;
    case 4: ok = launch_fwd_g<N, T, 4>(a, tw, st); break;
    case 8: ok = launch_fwd_g<N, T, 8>(a, tw, st); break;
  }
  if (!ok) {
    set_error("search: %d planes per CTA not available for box %d", g, N);
    return EMC_E_ARG;
  }
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

// Launches the three passes of one chunk with g planes per pass-A CTA; ev (optional) receives
// an event record before each pass and after the last one (4 events).
template <int N, typename T>
static emc_status launch_chunk(int g, const SearchChunkArgs& a, cudaStream_t st, cudaEvent_t* ev) {
  using C = SearchCfg<N>;
  const float2* tw = device_twiddles(N);
  if (!tw) return EMC_E_CUDA;
  const int w = 2 * a.radius + 1;
  if (ev) EMC_CUDA(cudaEventRecord(ev[0], st));
  EMC_TRY((launch_fwd<N, T>(g, a, tw, st)));
  if (ev) EMC_CUDA(cudaEventRecord(ev[1], st));
  k_search_z_mul<N><<<dim3(C::GRID_BX, (a.n_items + C::EVALS_B - 1) / C::EVALS_B), C::NT_B, C::SMEM_B, st>>>(a, tw);
  EMC_LAUNCH_CHECK();
  if (ev) EMC_CUDA(cudaEventRecord(ev[2], st));
  k_search_inv_peak<N><<<dim3(w, a.n_items), C::NT_BC, C::SMEM_C, st>>>(a, tw);
  EMC_LAUNCH_CHECK();
  if (ev) EMC_CUDA(cudaEventRecord(ev[3], st));
  return EMC_OK;
}

static bool box_supported(int n) { return n == 64 || n == 96 || n == 128; }

static int box_index(int n) { return n == 64 ? 0 : (n == 96 ? 1 : 2); }

template <int N>
static bool planes_fit_rt(int g) {
  switch (g) {
    case 1: return planes_fit<N, 1>();
    case 2: return planes_fit<N, 2>();
    case 4: return planes_fit<N, 4>();
    case 8: return planes_fit<N, 8>();
  }
  return false;
}

// Whether pass A can run box n with g planes per CTA (g divides n, the slab fits shared memory).
static bool planes_available(int n, int g) {
  switch (n) {
    case 64: return planes_fit_rt<64>(g);
    case 96: return planes_fit_rt<96>(g);
    case 128: return planes_fit_rt<128>(g);
  }
  return false;
}

template <typename T>
static emc_status launch_fwd_any_t(int n, int g, const SearchChunkArgs& a, cudaStream_t st) {
  const float2* tw = device_twiddles(n);
  if (!tw) return EMC_E_CUDA;
  switch (n) {
    case 64: return launch_fwd<64, T>(g, a, tw, st);
    case 96: return launch_fwd<96, T>(g, a, tw, st);
    case 128: return launch_fwd<128, T>(g, a, tw, st);
  }
  set_error("search: box %d not supported (64, 96, 128)", n);
  return EMC_E_UNSUPPORTED;
}

static emc_status launch_fwd_any(int n, int dtype, int g, const SearchChunkArgs& a, cudaStream_t st) {
  return dtype == EMC_DTYPE_F32 ? launch_fwd_any_t<float>(n, g, a, st)
                                : launch_fwd_any_t<__nv_bfloat16>(n, g, a, st);
}

static emc_status launch_chunk_any(int n, int dtype, int g, const SearchChunkArgs& a, cudaStream_t st,
                                   cudaEvent_t* ev) {
  if (dtype == EMC_DTYPE_F32) {
    switch (n) {
      case 64: return launch_chunk<64, float>(g, a, st, ev);
      case 96: return launch_chunk<96, float>(g, a, st, ev);
      case 128: return launch_chunk<128, float>(g, a, st, ev);
    }
  } else {
    switch (n) {
      case 64: return launch_chunk<64, __nv_bfloat16>(g, a, st, ev);
      case 96: return launch_chunk<96, __nv_bfloat16>(g, a, st, ev);
      case 128: return launch_chunk<128, __nv_bfloat16>(g, a, st, ev);
    }
  }
  set_error("search: box %d not supported (64, 96, 128)", n);
  return EMC_E_UNSUPPORTED;
}

static emc_status set_attrs_any(int n, int dtype) {
  if (dtype == EMC_DTYPE_F32) {
    switch (n) {
      case 64: return set_attrs<64, float>();
      case 96: return set_attrs<96, float>();
      case 128: return set_attrs<128, float>();
    }
  } else {
    switch (n) {
      case 64: return set_attrs<64, __nv_bfloat16>();
      case 96: return set_attrs<96, __nv_bfloat16>();
      case 128: return set_attrs<128, __nv_bfloat16>();
    }
  }
  return EMC_E_UNSUPPORTED;
}

static size_t per_eval_scratch(int n, int radius) {
  return sizeof(float2) * (s1_eval_elems(n) + s2_plane_elems(n) * (size_t)(2 * radius + 1));
}

// Device buffer that grows on demand.
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t cap = 0;
  emc_status reserve(size_t n) {
    if (n <= cap) return EMC_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1)) != cudaSuccess) {
      set_error("search: cudaMalloc(%zu) failed", sizeof(T) * n);
      return EMC_E_OOM;
    }
    cap = n;
    return EMC_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

// Weights particle blockIdx.y of a batch (spectra, weights and energies advance by nhalf, nhalf and
// 1 per particle; wgt_stride 0 shares one weight) and accumulates its energy.
__global__ void k_particle_weight(float2* __restrict__ q, const float* __restrict__ wgt, const float* __restrict__ bp,
                                  long nhalf, int nh, int n, double* __restrict__ energy, long wgt_stride = 0) {
  __shared__ double red[32];
  q += (long)blockIdx.y * nhalf;
  if (wgt) wgt += (long)blockIdx.y * wgt_stride;
  energy += blockIdx.y;
  double e = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nhalf; i += (long)gridDim.x * blockDim.x) {
    float f = 1.f;
    if (wgt) f *= wgt[i];
    if (bp) f *= bp[i];
    if (i == 0) f = 0.f;
    float2 v = q[i];
    v.x *= f;
    v.y *= f;
    q[i] = v;
    const int kx = (int)(i % nh);
    e += (kx == 0 || 2 * kx == n ? 1.0 : 2.0) * ((double)v.x * v.x + (double)v.y * v.y);
  }
  double t = block_sum(e, red);
  if (threadIdx.x == 0) atomicAdd(energy, t);
}

}  // namespace emc

// ===================================================================== C-ABI
struct emc_search_s {
  struct Ref {
    void* data = nullptr;
    float* mask = nullptr;
    float* wref = nullptr;
    void* cells = nullptr;
    unsigned* mask_rows = nullptr;
    int n = 0;
    int dtype = 0;
  };
  std::vector<Ref> refs;
  emc::DevBuf<emc::DevRef> d_refs;
  bool refs_dirty = true;
  std::vector<double> dmat;  // [norient][9]
  emc::DevBuf<double> d_dmat;
  int norient = 0;
  int radius = 0, interp = EMC_INTERP_LINEAR, chunk_evals = 0;
  // S1 + S2 scratch of a chunk: 768 MiB (about 600 evaluations at 64^3, 190 at 96^3, 84 at 128^3 with
  // radius 7), or an eighth of the free device memory if that is less.  Measured: evaluations/s rise
  // with the chunk until about this size (64^3: 370 k at 66 evaluations, the two-thirds-of-L2
  // sizing, 400 k at 592, 403 k at 888; 96^3: 80 k at 21, 88 k at 168; 128^3: 31 k at 9, 34 k at
  // 72): larger chunks amortise the passes' launch tails, and the slabs that then spill from L2
  // cost HBM bandwidth the passes leave unused
  size_t scratch_budget = 768ull << 20;

  // Particle table and evaluation list of one recorded request.  Each cached graph reads its own
  // (the graph replays kernels that read them), so alternating requests -- a double-buffered
  // pipeline whose descriptors point at one of two input buffers -- replay instead of re-recording.
  struct RunTables {
    emc::DevBuf<emc::DevParticle> parts;
    emc::DevBuf<emc::EvalItem> items;
    void release() {
      parts.release();
      items.release();
    }
  };
  struct GraphEntry {
    std::vector<char> key;
    cudaGraphExec_t exec = nullptr;
    RunTables tables;
    unsigned long long used = 0;
  };
  static constexpr size_t kGraphCache = 4;
  std::vector<GraphEntry> graphs;  // least recently used evicted; capacity reserved at creation
  unsigned long long use_clock = 0;
  RunTables eager_tables;          // tables of profiled (eager, unrecorded) runs
  RunTables* cur = nullptr;        // tables of the run being recorded or launched eagerly
  emc::DevBuf<emc::EvalResult> d_results;
  emc::DevBuf<unsigned long long> d_best_keys;
  // device status word of bounded waits (emc::kStatusWaitTimeout), read and cleared by
  // emc_search_status and emc_search_run_host; the wait limit and the test hook's phantom bytes
  emc::DevBuf<unsigned> d_status;
  // device outputs of emc_search_run_host, kept between calls (grown on demand) so that a repeated
  // request replays its recorded graph
  emc::DevBuf<float> host_cc;
  emc::DevBuf<int> host_peak;
  emc::DevBuf<emc_search_hit> host_best;
  long long wait_cycles = 1ll << 31;
  unsigned phantom_tx = 0;
  // Per-evaluation scratch of a chunk, one set per overlap slot: chunk i of a recorded run uses slot
  // i % overlap and its own branch of the graph, so consecutive chunks run concurrently (pass A of one
  // beside passes B and C of the other, filling each other's tails) while chunks of one slot stay in order.
  static constexpr int kMaxSlots = 2;
  struct Scratch {
    emc::DevBuf<float2> s1, s2;
    emc::DevBuf<emc::EvalStats> stats;
    emc::DevBuf<unsigned long long> keys;
    emc::DevBuf<unsigned> done;
    void release() {
      s1.release();
      s2.release();
      stats.release();
      keys.release();
      done.release();
    }
  };
  Scratch slot[kMaxSlots];
  int overlap = kMaxSlots;        // slots used by recorded runs (profiled runs use one)
  cudaStream_t branch = nullptr;  // the second branch's stream during capture
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;

  const double* run_energy = nullptr;  // device energies of the run being recorded (or null)
  cudaStream_t cap_stream = nullptr;
  long last_launches = 0;

  // profiling: a ring of per-chunk event sets, harvested before reuse
  bool profiling = false;
  static constexpr int kRing = 64;
  cudaEvent_t ev[kRing][5] = {};
  bool ev_pending[kRing] = {};
  int ev_next = 0;
  double prof_ms[4] = {0, 0, 0, 0};
  long prof_launches[4] = {0, 0, 0, 0};
  long prof_evals = 0;

  // pass-A planes per CTA per [box 64/96/128][dtype]: 0 = tune on the next run
  int planes[3][2] = {};
  float tune_ms[3][2][4] = {{{-1, -1, -1, -1}, {-1, -1, -1, -1}},
                            {{-1, -1, -1, -1}, {-1, -1, -1, -1}},
                            {{-1, -1, -1, -1}, {-1, -1, -1, -1}}};
};

namespace {

struct Chunk {
  int n, dtype;
  long item_offset;
  int count;
};

int effective_radius(const emc_search_s* s, int n) {
  int r = s->radius > 0 ? s->radius : std::max(1, n / 8);
  return std::min(r, n / 2 - 1);
}

// Forgets every recorded request (their graphs hold scratch pointers and read the orientation and
// reference tables, so any change to those invalidates them).
void drop_graphs(emc_search_s* s) {
  for (auto& g : s->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.tables.release();
  }
  s->graphs.clear();
}

}  // namespace

extern "C" {

emc_status emc_search_create(emc_search_t* out) {
  EMC_CHECK_ARG(out, "emc_search_create: null argument");
  emc_search_s* s = new (std::nothrow) emc_search_s();
  EMC_CHECK_ARG(s, "emc_search_create: host allocation failed");
  {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && free_b / 8 < s->scratch_budget)
      s->scratch_budget = std::max<size_t>(free_b / 8, 16ull << 20);
  }
  s->graphs.reserve(emc_search_s::kGraphCache);
  if (s->d_status.reserve(1) != EMC_OK || cudaMemset(s->d_status.p, 0, sizeof(unsigned)) != cudaSuccess) {
    delete s;
    emc::set_error("emc_search_create: status word allocation failed");
    return EMC_E_OOM;
  }
  if (cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->branch, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->join_ev, cudaEventDisableTiming) != cudaSuccess) {
    if (s->cap_stream) cudaStreamDestroy(s->cap_stream);
    if (s->branch) cudaStreamDestroy(s->branch);
    if (s->fork_ev) cudaEventDestroy(s->fork_ev);
    if (s->join_ev) cudaEventDestroy(s->join_ev);
    delete s;
    emc::set_error("emc_search_create: stream or event creation failed");
    return EMC_E_CUDA;
  }
  *out = s;
  return EMC_OK;
}

emc_status emc_search_add_reference(emc_search_t s, const float* d_ref, int n, const float* d_mask, const float* d_wref,
                                    int store_dtype, int* ref_id, void* stream) {
  EMC_CHECK_ARG(s && d_ref && ref_id, "emc_search_add_reference: null argument");
  EMC_CHECK_ARG(emc::box_supported(n), "emc_search_add_reference: box %d not supported (64, 96, 128)", n);
  EMC_CHECK_ARG(store_dtype == EMC_DTYPE_F32 || store_dtype == EMC_DTYPE_BF16, "emc_search_add_reference: dtype");
  cudaStream_t st = emc::as_stream(stream);
  emc_search_s::Ref r;
  r.n = n;
  r.dtype = store_dtype;
  const long nv = (long)n * n * n, nhalf = (long)(n / 2 + 1) * n * n;
  const size_t vb = nv * (store_dtype == EMC_DTYPE_F32 ? 4 : 2);
  EMC_CUDA(cudaMalloc(&r.data, vb));
  if (store_dtype == EMC_DTYPE_F32) {
    EMC_CUDA(cudaMemcpyAsync(r.data, d_ref, vb, cudaMemcpyDeviceToDevice, st));
  } else {
    EMC_TRY(emc::to_bf16(d_ref, reinterpret_cast<__nv_bfloat16*>(r.data), nv, st));
  }
  if (d_mask) {
    EMC_CUDA(cudaMalloc(&r.mask, nv * sizeof(float)));
    EMC_CUDA(cudaMemcpyAsync(r.mask, d_mask, nv * sizeof(float), cudaMemcpyDeviceToDevice, st));
    // each row's x extent of non-zero mask voxels: the gather skips the cells outside it
    EMC_CUDA(cudaMalloc(&r.mask_rows, sizeof(unsigned) * (size_t)n * n));
    emc::k_mask_rows<<<(n * n + 7) / 8, 256, 0, st>>>(r.mask, n, r.mask_rows);
    EMC_LAUNCH_CHECK();
  }
  if (d_wref) {
    EMC_CUDA(cudaMalloc(&r.wref, nhalf * sizeof(float)));
    EMC_CUDA(cudaMemcpyAsync(r.wref, d_wref, nhalf * sizeof(float), cudaMemcpyDeviceToDevice, st));
  }
  {
    // trilinear corner cells for the linear interpolation modes
    const long nc = (long)(n + 1) * (n + 1) * (n + 1);
    const int blocks = (int)std::min<long>((nc + 255) / 256, 4L * emc::device_sm_count());
    if (store_dtype == EMC_DTYPE_F32) {
      EMC_CUDA(cudaMalloc(&r.cells, nc * sizeof(emc::CellT<float>)));
      emc::k_build_cells<float><<<blocks, 256, 0, st>>>(d_ref, n, (emc::CellT<float>*)r.cells);
    } else {
      EMC_CUDA(cudaMalloc(&r.cells, nc * sizeof(emc::CellT<__nv_bfloat16>)));
      emc::k_build_cells<__nv_bfloat16><<<blocks, 256, 0, st>>>(d_ref, n, (emc::CellT<__nv_bfloat16>*)r.cells);
    }
    EMC_LAUNCH_CHECK();
  }
  EMC_TRY(emc::set_attrs_any(n, store_dtype));
  if (!emc::device_twiddles(n)) return EMC_E_CUDA;
  s->refs.push_back(r);
  s->refs_dirty = true;
  *ref_id = (int)s->refs.size() - 1;
  return EMC_OK;
}

emc_status emc_search_set_orientations(emc_search_t s, const double* ptp, int n) {
  EMC_CHECK_ARG(s && ptp && n > 0, "emc_search_set_orientations: bad argument");
  s->dmat.assign((size_t)n * 9, 0.0);
  for (int o = 0; o < n; ++o) {
    const double ang[3] = {ptp[3 * o], ptp[3 * o + 1], ptp[3 * o + 2] - ptp[3 * o]};
    EMC_TRY(emc_define_matrix(ang, 1, &s->dmat[(size_t)o * 9]));
  }
  EMC_TRY(s->d_dmat.reserve(s->dmat.size()));
  EMC_CUDA(cudaMemcpy(s->d_dmat.p, s->dmat.data(), sizeof(double) * s->dmat.size(), cudaMemcpyHostToDevice));
  s->norient = n;
  drop_graphs(s);
  return EMC_OK;
}

emc_status emc_search_configure(emc_search_t s, int peak_radius, int interp, int chunk_evals) {
  EMC_CHECK_ARG(s, "emc_search_configure: null handle");
  EMC_CHECK_ARG(peak_radius >= 0 && peak_radius < 64, "emc_search_configure: peak radius %d", peak_radius);
  EMC_CHECK_ARG(interp >= 0 && interp <= 2, "emc_search_configure: interp %d", interp);
  EMC_CHECK_ARG(chunk_evals >= 0, "emc_search_configure: chunk_evals %d", chunk_evals);
  s->radius = peak_radius;
  s->interp = interp;
  s->chunk_evals = chunk_evals;
  drop_graphs(s);
  return EMC_OK;
}

// Adds the elapsed times of a finished event set to the profile totals.
static emc_status harvest_slot(emc_search_t s, int slot) {
  if (!s->ev_pending[slot]) return EMC_OK;
  EMC_CUDA(cudaEventSynchronize(s->ev[slot][4]));
  for (int k = 0; k < 4; ++k) {
    float ms = 0.f;
    EMC_CUDA(cudaEventElapsedTime(&ms, s->ev[slot][k], s->ev[slot][k + 1]));
    s->prof_ms[k] += ms;
  }
  s->ev_pending[slot] = false;
  return EMC_OK;
}

static emc::SearchChunkArgs chunk_args(emc_search_t s, const Chunk& c, int slot = 0) {
  const emc_search_s::Scratch& sc = s->slot[slot];
  emc::SearchChunkArgs a;
  a.items = s->cur->items.p + c.item_offset;
  a.parts = s->cur->parts.p;
  a.refs = s->d_refs.p;
  a.dmat = s->d_dmat.p;
  a.s1 = sc.s1.p;
  a.s2 = sc.s2.p;
  a.stats = sc.stats.p;
  a.keys = sc.keys.p;
  a.n_items = c.count;
  a.radius = effective_radius(s, c.n);
  a.interp = s->interp;
  a.done = sc.done.p;
  a.results = s->d_results.p;
  a.best_keys = s->d_best_keys.p;
  a.status = s->d_status.p;
  a.wait_cycles = s->wait_cycles;
  a.phantom_tx = s->phantom_tx;
  return a;
}

// Reads and clears the status word (the stream synchronised by the caller).
static emc_status take_status(emc_search_t s) {
  unsigned v = 0;
  EMC_CUDA(cudaMemcpy(&v, s->d_status.p, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (!v) return EMC_OK;
  EMC_CUDA(cudaMemset(s->d_status.p, 0, sizeof(unsigned)));
  emc::set_error("search: a device-side wait for bulk copies gave up; that run's results are invalid");
  return EMC_E_TIMEOUT;
}

static int& planes_slot(emc_search_t s, int n, int dtype) {
  return s->planes[emc::box_index(n)][dtype == EMC_DTYPE_BF16 ? 1 : 0];
}

// Times pass A on chunk c with every planes option that fits (one warm-up launch, then three
// timed ones each) and stores the fastest. Pass A's outputs (S1 slabs, energy sums) are scratch
// that the real run rewrites, so the trial launches leave no trace in the results.
static emc_status tune_planes(emc_search_t s, const Chunk& c, cudaStream_t st) {
  const emc::SearchChunkArgs a = chunk_args(s, c);
  float* ms_out = s->tune_ms[emc::box_index(c.n)][c.dtype == EMC_DTYPE_BF16 ? 1 : 0];
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  EMC_CUDA(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    emc::set_error("search: event creation failed");
    return EMC_E_CUDA;
  }
  emc_status rs = EMC_OK;
  int best = 0;
  float best_ms = 0.f;
  constexpr int kReps = 3;
  for (int k = 0; k < 4 && rs == EMC_OK; ++k) {
    const int g = emc::kPlaneOptions[k];
    ms_out[k] = -1.f;
    if (!emc::planes_available(c.n, g)) continue;
    rs = emc::launch_fwd_any(c.n, c.dtype, g, a, st);
    if (rs == EMC_OK && cudaEventRecord(e0, st) != cudaSuccess) rs = EMC_E_CUDA;
    for (int r = 0; r < kReps && rs == EMC_OK; ++r) rs = emc::launch_fwd_any(c.n, c.dtype, g, a, st);
    float ms = 0.f;
    if (rs == EMC_OK && (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                         cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
      rs = EMC_E_CUDA;
    if (rs != EMC_OK) break;
    ms_out[k] = ms / kReps;
    if (!best || ms < best_ms) {
      best = g;
      best_ms = ms;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rs == EMC_E_CUDA) emc::set_error("search: pass-A tuning failed: %s", cudaGetErrorString(cudaGetLastError()));
  if (rs != EMC_OK) return rs;
  planes_slot(s, c.n, c.dtype) = best;
  return EMC_OK;
}

static emc_status search_record(emc_search_t s, const std::vector<Chunk>& chunks, int np, long total_evals,
                                float* d_cc, int* d_peak, emc_search_hit* d_best, cudaStream_t st) {
  EMC_CUDA(cudaMemsetAsync(s->d_best_keys.p, 0, sizeof(unsigned long long) * np, st));
  // per-evaluation scratch starts clear; the last pass-C CTA of each evaluation clears it again
  const int nslots = s->profiling ? 1 : s->overlap;
  for (int k = 0; k < nslots; ++k) {
    emc_search_s::Scratch& sc = s->slot[k];
    EMC_CUDA(cudaMemsetAsync(sc.stats.p, 0, sizeof(emc::EvalStats) * sc.stats.cap, st));
    EMC_CUDA(cudaMemsetAsync(sc.keys.p, 0, sizeof(unsigned long long) * sc.keys.cap, st));
    EMC_CUDA(cudaMemsetAsync(sc.done.p, 0, sizeof(unsigned) * sc.done.cap, st));
  }
  long launches = 0;
  if (s->run_energy) {
    emc::k_search_energies<<<(np + 255) / 256, 256, 0, st>>>(s->cur->parts.p, np, s->run_energy);
    EMC_LAUNCH_CHECK();
    ++launches;
  }
  // The second branch forks from the stream after the set-up above and joins before the outputs.
  // Only 64^3 chunks overlap; larger ones run alone on the stream (the branch joined first): their
  // passes fill the SMs by themselves, and beside another chunk's they ran slower (96^3: 96.0k
  // evaluations/s with two slots against 101.1k with one; 128^3: 40.2k against 44.9k).
  const bool two = nslots > 1 && chunks.size() > 1;
  bool forked = false;
  long alternate = 0;
  for (size_t ci = 0; ci < chunks.size(); ++ci) {
    const Chunk& c = chunks[ci];
    const bool overlapped = two && c.n <= 64;
    if (overlapped && !forked) {
      EMC_CUDA(cudaEventRecord(s->fork_ev, st));
      EMC_CUDA(cudaStreamWaitEvent(s->branch, s->fork_ev, 0));
      forked = true;
    } else if (!overlapped && forked) {
      EMC_CUDA(cudaEventRecord(s->join_ev, s->branch));
      EMC_CUDA(cudaStreamWaitEvent(st, s->join_ev, 0));
      forked = false;
    }
    const int slot = overlapped ? (int)(alternate++ % 2) : 0;
    const cudaStream_t cst = slot ? s->branch : st;
    const emc::SearchChunkArgs a = chunk_args(s, c, slot);
    cudaEvent_t* ev = nullptr;
    if (s->profiling) {
      const int slot = s->ev_next;
      s->ev_next = (s->ev_next + 1) % emc_search_s::kRing;
      EMC_TRY(harvest_slot(s, slot));
      ev = s->ev[slot];
      s->ev_pending[slot] = true;
    }
    EMC_TRY(emc::launch_chunk_any(c.n, c.dtype, planes_slot(s, c.n, c.dtype), a, cst, ev));
    if (ev) EMC_CUDA(cudaEventRecord(ev[4], cst));  // decode runs inside pass C
    launches += 3;
    if (s->profiling) {
      for (int k = 0; k < 4; ++k) s->prof_launches[k] += 1;
      s->prof_evals += c.count;
    }
  }
  if (forked) {
    EMC_CUDA(cudaEventRecord(s->join_ev, s->branch));
    EMC_CUDA(cudaStreamWaitEvent(st, s->join_ev, 0));
  }
  if (d_best) {
    emc::k_search_best<<<(np + 127) / 128, 128, 0, st>>>(s->cur->parts.p, np, s->d_results.p, s->d_best_keys.p, d_best);
    EMC_LAUNCH_CHECK();
    ++launches;
  }
  if (d_cc || d_peak) {
    const int blocks = (int)std::min<long>((total_evals + 255) / 256, 4L * emc::device_sm_count());
    emc::k_search_scatter<<<std::max(blocks, 1), 256, 0, st>>>(s->d_results.p, total_evals, d_cc, d_peak);
    EMC_LAUNCH_CHECK();
    ++launches;
  }
  s->last_launches = launches;
  return EMC_OK;
}

static emc_status search_run(emc_search_t s, const emc_particle_desc* particles, int np, const double* d_energy,
                             float* d_cc, int* d_peak, emc_search_hit* d_best, void* stream) {
  EMC_CHECK_ARG(s && particles && np > 0, "emc_search_run: bad argument");
  EMC_CHECK_ARG(s->norient > 0, "emc_search_run: no orientations set");
  cudaStream_t st = emc::as_stream(stream);
  // ---- validate and build the particle table
  std::vector<emc::DevParticle> parts(np);
  long total = 0;
  for (int p = 0; p < np; ++p) {
    const emc_particle_desc& d = particles[p];
    EMC_CHECK_ARG(d.spectrum, "particle %d: null spectrum", p);
    EMC_CHECK_ARG(d.ref_id >= 0 && d.ref_id < (int)s->refs.size(), "particle %d: bad ref_id %d", p, d.ref_id);
    EMC_CHECK_ARG(s->refs[d.ref_id].n == d.box, "particle %d: box %d does not match reference box %d", p, d.box,
                  s->refs[d.ref_id].n);
    EMC_CHECK_ARG(d.orient_begin >= 0 && d.orient_count >= 0 && d.orient_begin + d.orient_count <= s->norient,
                  "particle %d: orientation slice [%d, %d) outside [0, %d)", p, d.orient_begin,
                  d.orient_begin + d.orient_count, s->norient);
    EMC_CHECK_ARG(d_energy || d.energy > 0.0, "particle %d: energy must be > 0", p);
    emc::DevParticle& q = parts[p];
    q.spec = reinterpret_cast<const float2*>(d.spectrum);
    q.wedge = d.wedge;
    q.energy = d.energy;
    memcpy(q.prior, d.prior, sizeof(q.prior));
    memcpy(q.shift, d.shift, sizeof(q.shift));
    q.ref = d.ref_id;
    q.box = d.box;
    q.orient_begin = d.orient_begin;
    q.eval_base = total;
    total += d.orient_count;
  }
  EMC_CHECK_ARG(total > 0, "emc_search_run: no (particle, orientation) pairs");
  // ---- cache key: request content + outputs + settings
  std::vector<char> key(sizeof(emc_particle_desc) * np + 64);
  memcpy(key.data(), particles, sizeof(emc_particle_desc) * np);
  {
    char* k = key.data() + sizeof(emc_particle_desc) * np;
    memcpy(k, &d_cc, 8); memcpy(k + 8, &d_peak, 8); memcpy(k + 16, &d_best, 8);
    memcpy(k + 24, &s->radius, 4); memcpy(k + 28, &s->interp, 4); memcpy(k + 32, &s->chunk_evals, 4);
    memcpy(k + 36, &s->norient, 4);
    const size_t nref = s->refs.size();
    memcpy(k + 40, &nref, 8);
    memcpy(k + 48, &st, 8);
    memcpy(k + 56, &d_energy, 8);
  }
  s->run_energy = d_energy;
  if (s->refs_dirty) drop_graphs(s);
  if (!s->profiling) {
    for (auto& g : s->graphs)
      if (g.key == key) {
        g.used = ++s->use_clock;
        EMC_CUDA(cudaGraphLaunch(g.exec, st));
        return EMC_OK;
      }
  }
  // ---- group pairs by (box, dtype) and cut chunks
  std::vector<emc::EvalItem> items;
  items.reserve(total);
  std::vector<Chunk> chunks;
  size_t max_chunk_bytes = 0;
  int max_chunk = 0;
  for (int n : {64, 96, 128})
    for (int dt : {EMC_DTYPE_F32, EMC_DTYPE_BF16}) {
      const long begin = (long)items.size();
      for (int p = 0; p < np; ++p) {
        if (particles[p].box != n || s->refs[particles[p].ref_id].dtype != dt) continue;
        for (int k = 0; k < particles[p].orient_count; ++k) items.push_back({p, particles[p].orient_begin + k});
      }
      const long cnt = (long)items.size() - begin;
      if (!cnt) continue;
      const int r = effective_radius(s, n);
      const size_t pe = emc::per_eval_scratch(n, r);
      const bool auto_size = s->chunk_evals <= 0;
      int e = auto_size ? (int)std::max<size_t>(1, s->scratch_budget / pe) : s->chunk_evals;
      e = (int)std::min<long>(e, 65535);
      if (auto_size) {
        // chunks of equal size (520 + 20 evaluations left the second overlap slot idle), and at least
        // two at 64^3, whose chunks overlap in pairs
        long k = (cnt + e - 1) / e;
        if (n <= 64 && s->overlap > 1 && cnt >= 64) k = std::max(k, 2L);
        e = (int)((cnt + k - 1) / k);
      }
      for (long off = 0; off < cnt; off += e) {
        Chunk c{n, dt, begin + off, (int)std::min<long>(e, cnt - off)};
        chunks.push_back(c);
        max_chunk_bytes = std::max(max_chunk_bytes, pe * c.count);
        max_chunk = std::max(max_chunk, c.count);
      }
    }
  // ---- shared scratch (a reallocation invalidates every recorded request)
  const int nslots = s->profiling ? 1 : s->overlap;
  auto scratch_ptrs = [&](std::vector<const void*>& v) {
    v = {s->d_results.p, s->d_best_keys.p};
    for (int k = 0; k < emc_search_s::kMaxSlots; ++k) {
      const emc_search_s::Scratch& sc = s->slot[k];
      v.insert(v.end(), {sc.stats.p, sc.keys.p, sc.done.p, sc.s1.p, sc.s2.p});
    }
  };
  std::vector<const void*> before, after;
  scratch_ptrs(before);
  EMC_TRY(s->d_results.reserve(total));
  EMC_TRY(s->d_best_keys.reserve(np));
  for (int k = 0; k < nslots; ++k) {
    EMC_TRY(s->slot[k].stats.reserve(max_chunk));
    EMC_TRY(s->slot[k].keys.reserve(max_chunk));
    EMC_TRY(s->slot[k].done.reserve(max_chunk));
  }
  {
    // split scratch between S1 and S2 proportionally to the largest chunk of each size
    size_t s1n = 0, s2n = 0;
    for (const Chunk& c : chunks) {
      const int r = effective_radius(s, c.n);
      s1n = std::max(s1n, (size_t)c.count * emc::s1_eval_elems(c.n));
      s2n = std::max(s2n, (size_t)c.count * (2 * r + 1) * emc::s2_plane_elems(c.n));
    }
    for (int k = 0; k < nslots; ++k) {
      EMC_TRY(s->slot[k].s1.reserve(s1n));
      EMC_TRY(s->slot[k].s2.reserve(s2n));
    }
  }
  scratch_ptrs(after);
  if (before != after) drop_graphs(s);
  if (s->refs_dirty) {
    std::vector<emc::DevRef> dr(s->refs.size());
    for (size_t i = 0; i < s->refs.size(); ++i)
      dr[i] = {s->refs[i].data, s->refs[i].mask,  s->refs[i].wref,     s->refs[i].n,
               s->refs[i].dtype, s->refs[i].cells, s->refs[i].mask_rows};
    EMC_TRY(s->d_refs.reserve(dr.size()));
    EMC_CUDA(cudaMemcpy(s->d_refs.p, dr.data(), sizeof(emc::DevRef) * dr.size(), cudaMemcpyHostToDevice));
    s->refs_dirty = false;
  }
  // ---- this request's tables: the eager set when profiling, else a new cache entry
  emc_search_s::GraphEntry* entry = nullptr;
  if (s->profiling) {
    s->cur = &s->eager_tables;
  } else {
    if (s->graphs.size() >= emc_search_s::kGraphCache) {
      auto lru = std::min_element(s->graphs.begin(), s->graphs.end(),
                                  [](const auto& a, const auto& b) { return a.used < b.used; });
      if (lru->exec) cudaGraphExecDestroy(lru->exec);
      lru->tables.release();
      s->graphs.erase(lru);
    }
    s->graphs.emplace_back();
    entry = &s->graphs.back();
    s->cur = &entry->tables;
  }
  auto abandon = [&](emc_status rs) {
    if (entry) {
      entry->tables.release();
      s->graphs.pop_back();
    }
    return rs;
  };
  {
    emc_status rs = s->cur->parts.reserve(np);
    if (rs == EMC_OK) rs = s->cur->items.reserve(items.size());
    if (rs != EMC_OK) return abandon(rs);
  }
  if (cudaMemcpyAsync(s->cur->parts.p, parts.data(), sizeof(emc::DevParticle) * np, cudaMemcpyHostToDevice, st) ||
      cudaMemcpyAsync(s->cur->items.p, items.data(), sizeof(emc::EvalItem) * items.size(), cudaMemcpyHostToDevice,
                      st) ||
      // host vectors must outlive the async copies
      cudaStreamSynchronize(st)) {
    emc::set_error("emc_search_run: table upload failed: %s", cudaGetErrorString(cudaGetLastError()));
    return abandon(EMC_E_CUDA);
  }
  for (const Chunk& c : chunks)
    if (!planes_slot(s, c.n, c.dtype)) {
      const emc_status rs = tune_planes(s, c, st);
      if (rs != EMC_OK) return abandon(rs);
    }
  if (s->profiling) return search_record(s, chunks, np, total, d_cc, d_peak, d_best, st);
  // ---- capture the launch sequence into a graph, then launch it
  if (cudaStreamBeginCapture(s->cap_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    emc::set_error("emc_search_run: stream capture failed to start");
    return abandon(EMC_E_CUDA);
  }
  emc_status rs = search_record(s, chunks, np, total, d_cc, d_peak, d_best, s->cap_stream);
  cudaGraph_t graph = nullptr;
  cudaError_t ce = cudaStreamEndCapture(s->cap_stream, &graph);
  if (rs != EMC_OK) {
    if (graph) cudaGraphDestroy(graph);
    return abandon(rs);
  }
  if (ce != cudaSuccess) {
    emc::set_error("emc_search_run: graph capture failed: %s", cudaGetErrorString(ce));
    return abandon(EMC_E_CUDA);
  }
  ce = cudaGraphInstantiate(&entry->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess) {
    emc::set_error("emc_search_run: graph instantiation failed: %s", cudaGetErrorString(ce));
    entry->exec = nullptr;
    return abandon(EMC_E_CUDA);
  }
  entry->key = key;
  entry->used = ++s->use_clock;
  EMC_CUDA(cudaGraphLaunch(entry->exec, st));
  return EMC_OK;
}

emc_status emc_search_run(emc_search_t s, const emc_particle_desc* particles, int np, float* d_cc, int* d_peak,
                          emc_search_hit* d_best, void* stream) {
  return search_run(s, particles, np, nullptr, d_cc, d_peak, d_best, stream);
}

emc_status emc_search_run_energies(emc_search_t s, const emc_particle_desc* particles, int np,
                                   const double* d_energy, float* d_cc, int* d_peak, emc_search_hit* d_best,
                                   void* stream) {
  EMC_CHECK_ARG(d_energy, "emc_search_run_energies: null energy array");
  return search_run(s, particles, np, d_energy, d_cc, d_peak, d_best, stream);
}

emc_status emc_search_run_host(emc_search_t s, const emc_particle_desc* particles, int np, float* h_cc, int* h_peak,
                               emc_search_hit* h_best, void* stream) {
  EMC_CHECK_ARG(s && particles && np > 0, "emc_search_run_host: bad argument");
  cudaStream_t st = emc::as_stream(stream);
  long total = 0;
  for (int p = 0; p < np; ++p) total += particles[p].orient_count;
  // the handle's output buffers: the stream's earlier work on them ended with the previous call's
  // synchronisation, so growing them here frees nothing in use
  emc_status rs = EMC_OK;
  if (h_cc) rs = s->host_cc.reserve((size_t)std::max<long>(total, 1));
  if (rs == EMC_OK && h_peak) rs = s->host_peak.reserve(3 * (size_t)std::max<long>(total, 1));
  if (rs == EMC_OK && h_best) rs = s->host_best.reserve((size_t)np);
  float* d_cc = h_cc ? s->host_cc.p : nullptr;
  int* d_peak = h_peak ? s->host_peak.p : nullptr;
  emc_search_hit* d_best = h_best ? s->host_best.p : nullptr;
  if (rs == EMC_OK) rs = emc_search_run(s, particles, np, d_cc, d_peak, d_best, stream);
  if (rs == EMC_OK && h_cc && cudaMemcpyAsync(h_cc, d_cc, sizeof(float) * total, cudaMemcpyDeviceToHost, st))
    rs = EMC_E_CUDA;
  if (rs == EMC_OK && h_peak &&
      cudaMemcpyAsync(h_peak, d_peak, sizeof(int) * 3 * total, cudaMemcpyDeviceToHost, st))
    rs = EMC_E_CUDA;
  if (rs == EMC_OK && h_best &&
      cudaMemcpyAsync(h_best, d_best, sizeof(emc_search_hit) * np, cudaMemcpyDeviceToHost, st))
    rs = EMC_E_CUDA;
  if (rs == EMC_OK && cudaStreamSynchronize(st) != cudaSuccess) rs = EMC_E_CUDA;
  if (rs == EMC_E_OOM) emc::set_error("emc_search_run_host: device allocation failed");
  if (rs == EMC_E_CUDA) emc::set_error("emc_search_run_host: copy back failed");
  if (rs == EMC_OK) rs = take_status(s);
  return rs;
}

emc_status emc_search_status(emc_search_t s, void* stream) {
  EMC_CHECK_ARG(s, "emc_search_status: null handle");
  EMC_CUDA(cudaStreamSynchronize(emc::as_stream(stream)));
  return take_status(s);
}

emc_status emc_search_test_wait(emc_search_t s, long long wait_cycles, unsigned phantom_bytes) {
  EMC_CHECK_ARG(s, "emc_search_test_wait: null handle");
  EMC_CHECK_ARG(wait_cycles > 0 && phantom_bytes % 16 == 0 && phantom_bytes <= 4096,
                "emc_search_test_wait: wait_cycles %lld > 0, phantom_bytes %u a multiple of 16 up to 4096",
                wait_cycles, phantom_bytes);
  s->wait_cycles = wait_cycles;
  s->phantom_tx = phantom_bytes;
  drop_graphs(s);  // recorded graphs hold the old values
  return EMC_OK;
}

emc_status emc_search_set_profiling(emc_search_t s, int enable) {
  EMC_CHECK_ARG(s, "emc_search_set_profiling: null handle");
  if (enable && !s->ev[0][0]) {
    for (int i = 0; i < emc_search_s::kRing; ++i)
      for (int k = 0; k < 5; ++k) EMC_CUDA(cudaEventCreate(&s->ev[i][k]));
  }
  s->profiling = enable != 0;
  return EMC_OK;
}

emc_status emc_search_timings(emc_search_t s, double ms[4], long launches[4], long* evals, long* launches_last_run,
                              int reset) {
  EMC_CHECK_ARG(s, "emc_search_timings: null handle");
  for (int i = 0; i < emc_search_s::kRing; ++i) EMC_TRY(harvest_slot(s, i));
  for (int k = 0; k < 4; ++k) {
    if (ms) ms[k] = s->prof_ms[k];
    if (launches) launches[k] = s->prof_launches[k];
  }
  if (evals) *evals = s->prof_evals;
  if (launches_last_run) *launches_last_run = s->last_launches;
  if (reset) {
    for (int k = 0; k < 4; ++k) {
      s->prof_ms[k] = 0;
      s->prof_launches[k] = 0;
    }
    s->prof_evals = 0;
  }
  return EMC_OK;
}

emc_status emc_search_set_planes(emc_search_t s, int box, int planes) {
  EMC_CHECK_ARG(s, "emc_search_set_planes: null handle");
  EMC_CHECK_ARG(emc::box_supported(box), "emc_search_set_planes: box %d not supported (64, 96, 128)", box);
  EMC_CHECK_ARG(planes == 0 || emc::planes_available(box, planes),
                "emc_search_set_planes: %d planes per CTA not available for box %d", planes, box);
  const int b = emc::box_index(box);
  for (int d = 0; d < 2; ++d) {
    s->planes[b][d] = planes;
    for (int k = 0; k < 4; ++k) s->tune_ms[b][d][k] = -1.f;
  }
  drop_graphs(s);
  return EMC_OK;
}

emc_status emc_search_set_overlap(emc_search_t s, int slots) {
  EMC_CHECK_ARG(s, "emc_search_set_overlap: null handle");
  EMC_CHECK_ARG(slots >= 1 && slots <= emc_search_s::kMaxSlots, "emc_search_set_overlap: %d slots (1 or %d)", slots,
                emc_search_s::kMaxSlots);
  s->overlap = slots;
  drop_graphs(s);
  return EMC_OK;
}

emc_status emc_search_get_planes(emc_search_t s, int box, int dtype, int* planes, float ms_per_option[4]) {
  EMC_CHECK_ARG(s && planes, "emc_search_get_planes: null argument");
  EMC_CHECK_ARG(emc::box_supported(box), "emc_search_get_planes: box %d not supported (64, 96, 128)", box);
  EMC_CHECK_ARG(dtype == EMC_DTYPE_F32 || dtype == EMC_DTYPE_BF16, "emc_search_get_planes: dtype %d", dtype);
  const int b = emc::box_index(box), d = dtype == EMC_DTYPE_BF16 ? 1 : 0;
  *planes = s->planes[b][d];
  if (ms_per_option)
    for (int k = 0; k < 4; ++k) ms_per_option[k] = s->tune_ms[b][d][k];
  return EMC_OK;
}

emc_status emc_search_destroy(emc_search_t s) {
  if (!s) return EMC_OK;
  for (int i = 0; i < emc_search_s::kRing; ++i)
    for (int k = 0; k < 5; ++k)
      if (s->ev[i][k]) cudaEventDestroy(s->ev[i][k]);
  drop_graphs(s);
  s->eager_tables.release();
  for (auto& r : s->refs) {
    cudaFree(r.data);
    cudaFree(r.mask);
    cudaFree(r.wref);
    cudaFree(r.cells);
    cudaFree(r.mask_rows);
  }
  s->d_refs.release();
  s->d_dmat.release();
  s->d_results.release();
  s->d_best_keys.release();
  s->d_status.release();
  s->host_cc.release();
  s->host_peak.release();
  s->host_best.release();
  for (auto& sc : s->slot) sc.release();
  if (s->branch) cudaStreamDestroy(s->branch);
  if (s->fork_ev) cudaEventDestroy(s->fork_ev);
  if (s->join_ev) cudaEventDestroy(s->join_ev);
  if (s->cap_stream) cudaStreamDestroy(s->cap_stream);
  delete s;
  return EMC_OK;
}

emc_status emc_particle_spectrum(int n, const float* d_particle, const float* d_weight, const float* d_bandpass,
                                 float* d_spectrum_out, double* d_energy, void* stream) {
  EMC_CHECK_ARG(d_particle && d_spectrum_out && d_energy, "emc_particle_spectrum: null argument");
  EMC_CHECK_ARG(emc::fft_length_supported(n) && n >= 2, "emc_particle_spectrum: box %d not supported", n);
  cudaStream_t st = emc::as_stream(stream);
  float2* q = reinterpret_cast<float2*>(d_spectrum_out);
  EMC_TRY(emc::fft3_r2c(d_particle, q, n, n, n, 1, st));
  EMC_CUDA(cudaMemsetAsync(d_energy, 0, sizeof(double), st));
  const long nhalf = (long)(n / 2 + 1) * n * n;
  const int blocks = (int)std::min<long>((nhalf + 255) / 256, 2L * emc::device_sm_count());
  emc::k_particle_weight<<<blocks, 256, 0, st>>>(q, d_weight, d_bandpass, nhalf, n / 2 + 1, n, d_energy);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

emc_status emc_particle_spectra(int n, int count, const float* d_particles, const float* d_weights,
                                const float* d_bandpass, float* d_spectra_out, double* d_energies, void* stream) {
  EMC_CHECK_ARG(d_particles && d_spectra_out && d_energies && count > 0, "emc_particle_spectra: bad argument");
  EMC_CHECK_ARG(emc::fft_length_supported(n) && n >= 2, "emc_particle_spectra: box %d not supported", n);
  EMC_CHECK_ARG(count <= 65535, "emc_particle_spectra: at most 65535 particles per call (got %d)", count);
  cudaStream_t st = emc::as_stream(stream);
  float2* q = reinterpret_cast<float2*>(d_spectra_out);
  EMC_TRY(emc::fft3_r2c(d_particles, q, n, n, n, count, st));
  EMC_CUDA(cudaMemsetAsync(d_energies, 0, sizeof(double) * count, st));
  const long nhalf = (long)(n / 2 + 1) * n * n;
  const int bx = (int)std::max<long>(1, std::min<long>((nhalf + 255) / 256, (2L * emc::device_sm_count() + count - 1) / count));
  emc::k_particle_weight<<<dim3(bx, count), 256, 0, st>>>(q, d_weights, d_bandpass, nhalf, n / 2 + 1, n, d_energies,
                                                          nhalf);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

emc_status emc_particle_template(int n, const float* d_spectrum, float* d_h, void* stream) {
  EMC_CHECK_ARG(d_spectrum && d_h, "emc_particle_template: null argument");
  EMC_CHECK_ARG(emc::fft_length_supported(n) && n >= 2, "emc_particle_template: box %d not supported", n);
  cudaStream_t st = emc::as_stream(stream);
  const size_t nhalf = (size_t)(n / 2 + 1) * n * n;
  float2* scratch = nullptr;
  EMC_CUDA(cudaMallocAsync(&scratch, nhalf * sizeof(float2), st));
  emc_status rs = emc::fft3_c2r(reinterpret_cast<const float2*>(d_spectrum), d_h, scratch, n, n, n, 1, st);
  cudaFreeAsync(scratch, st);
  return rs;
}

}  // extern "C"

// Read access to a registered reference (used by the adjoint entry point).
emc_status emc_search_reference_info(emc_search_t s, int ref_id, const void** data, const void** cells,
                                     const float** mask, int* n, int* dtype) {
  EMC_CHECK_ARG(s && data && cells && mask && n && dtype, "emc_search_reference_info: null argument");
  EMC_CHECK_ARG(ref_id >= 0 && ref_id < (int)s->refs.size(), "reference id %d not registered", ref_id);
  const auto& r = s->refs[ref_id];
  *data = r.data;
  *cells = r.cells;
  *mask = r.mask;
  *n = r.n;
  *dtype = r.dtype;
  return EMC_OK;
}
