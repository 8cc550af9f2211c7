// search_noalloc.cu -- single-particle orientation search that never allocates device memory.
//
// Some callers cannot call cudaMalloc once they are running: hosts that hand the whole GPU to
// their own memory pool (MATLAB's gpuArray allocator, a framework's caching allocator) where a
// raw allocation can fail or fragment the pool, and processing loops that are only allowed to
// allocate at start-up so that their latency stays bounded.  emc_search_plain_noalloc serves
// them: the caller passes inputs and outputs, and every piece of scratch (the spilled spectra of
// the three passes, per-evaluation statistics and keys, the orientation matrices, the FFT twiddle
// tables) lives in one file-scope __device__ array of EMC_NOALLOC_SCRATCH_BYTES that each GPU
// holds from library load until process exit.
//
// The kernels are the same three passes as emc_search_run (search_kernels.cuh), launched
// directly on the caller's stream.
#include <math.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "search_kernels.cuh"

#define EMC_NOALLOC_SCRATCH_BYTES (24u << 20)  // 24 MiB per device
#define EMC_NOALLOC_MAX_ORIENT 4096
#define EMC_NOALLOC_MAX_RADIUS 15

namespace emc {
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[EMC_NOALLOC_SCRATCH_BYTES];

struct NoallocResult {
  float cc;
  int peak[3];
};

// Layout of the scratch array (byte offsets, every region 256-byte aligned).
constexpr size_t kTwOff = 0;                                              // twiddles 64 + 96 + 128
constexpr size_t kTwBytes = 256 * 8 * 2;
constexpr size_t kHdrOff = kTwOff + kTwBytes;                             // DevParticle + DevRef
constexpr size_t kHdrBytes = 512;
constexpr size_t kDmatOff = kHdrOff + kHdrBytes;                          // orientation matrices
constexpr size_t kDmatBytes = sizeof(double) * 9 * EMC_NOALLOC_MAX_ORIENT;
constexpr size_t kItemOff = kDmatOff + kDmatBytes;                        // EvalItem per orientation
constexpr size_t kItemBytes = sizeof(EvalItem) * EMC_NOALLOC_MAX_ORIENT;
constexpr size_t kResOff = kItemOff + kItemBytes;                         // per-orientation results
constexpr size_t kResBytes = sizeof(NoallocResult) * EMC_NOALLOC_MAX_ORIENT;
constexpr size_t kBestOff = kResOff + kResBytes;                          // best key, status word at +8
constexpr size_t kBestBytes = 256;
constexpr size_t kStatOff = kBestOff + kBestBytes;                        // stats + keys per chunk slot
constexpr size_t kMaxChunk = 64;
constexpr size_t kStatBytes = (sizeof(EvalStats) + sizeof(unsigned long long)) * kMaxChunk;
constexpr size_t kSpecOff = ((kStatOff + kStatBytes + 255) / 256) * 256;  // S1 then S2
static_assert(kSpecOff < EMC_NOALLOC_SCRATCH_BYTES, "scratch layout");
static_assert(kItemOff % 8 == 0 && kResOff % 16 == 0 && kStatOff % 16 == 0, "alignment");

struct DeviceState {
  unsigned char* base = nullptr;  // device address of g_noalloc_scratch
  bool ready = false;
};
constexpr int kMaxDev = 64;
DeviceState g_state[kMaxDev];
std::mutex g_mutex;

int tw_offset(int n) { return n == 64 ? 0 : (n == 96 ? 64 : 160); }

__global__ void k_noalloc_decode(const SearchChunkArgs a, int n, NoallocResult* __restrict__ res,
                                 unsigned long long* __restrict__ best) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.n_items) return;
  const int o = a.items[e].orient;
  const unsigned long long key = a.keys[e];
  NoallocResult r;
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
    atomicMax(best, ((unsigned long long)ordered_key(r.cc) << 32) | (0xffffffffu - (unsigned)o));
  }
  res[o] = r;
}

__global__ void k_noalloc_outputs(const NoallocResult* __restrict__ res, int n_orient,
                                  const unsigned long long* __restrict__ best, float* __restrict__ cc,
                                  int* __restrict__ peak, emc_search_hit* __restrict__ hit) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_orient) {
    const NoallocResult r = res[i];
    if (cc) cc[i] = r.cc;
    if (peak) { peak[3 * i] = r.peak[0]; peak[3 * i + 1] = r.peak[1]; peak[3 * i + 2] = r.peak[2]; }
  }
  if (i == 0 && hit) {
    emc_search_hit h;
    const unsigned long long k = *best;
    if (k == 0ull) {
      h.cc = __int_as_float(0x7fc00000);
      h.orient = -1;
      h.peak[0] = h.peak[1] = h.peak[2] = 0;
    } else {
      const int o = (int)(0xffffffffu - (unsigned int)(k & 0xffffffffull));
      h.cc = res[o].cc;
      h.orient = o;
      h.peak[0] = res[o].peak[0]; h.peak[1] = res[o].peak[1]; h.peak[2] = res[o].peak[2];
    }
    *hit = h;
  }
}

template <int N, typename T>
emc_status set_attrs_noalloc() {
  using C = SearchCfg<N>;
  EMC_CUDA(cudaFuncSetAttribute(k_search_fwd_xy<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM_A));
  EMC_CUDA(cudaFuncSetAttribute(k_search_z_mul<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM_B));
  EMC_CUDA(cudaFuncSetAttribute(k_search_inv_peak<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM_C));
  return EMC_OK;
}

// Once per device, with that device current: resolve the device address of the scratch array
// (its host-side name is only a stand-in), upload the twiddle tables on the caller's stream and wait
// for that stream (so no other thread's call on another stream can read them early, and the legacy
// default stream is not involved), set kernel attributes.  Under CUDA's lazy module loading the
// array itself is allocated when this first call loads the module.
emc_status setup_device(unsigned char** base, cudaStream_t stream) {
  int dev = 0;
  EMC_CUDA(cudaGetDevice(&dev));
  EMC_CHECK_ARG(dev >= 0 && dev < kMaxDev, "emc_search_plain_noalloc: device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_mutex);
  DeviceState& st = g_state[dev];
  if (!st.ready) {
    void* p = nullptr;
    EMC_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    std::vector<float2> tw(64 + 96 + 128);
    for (int n : {64, 96, 128})
      for (int m = 0; m < n; ++m) {
        const double a = -2.0 * M_PI * (double)m / (double)n;
        tw[tw_offset(n) + m] = make_float2((float)cos(a), (float)sin(a));
      }
    EMC_CUDA(cudaMemcpyAsync((unsigned char*)p + kTwOff, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice,
                             stream));
    EMC_CUDA(cudaStreamSynchronize(stream));
    EMC_TRY((set_attrs_noalloc<64, float>()));
    EMC_TRY((set_attrs_noalloc<96, float>()));
    EMC_TRY((set_attrs_noalloc<128, float>()));
    st.base = (unsigned char*)p;
    st.ready = true;
  }
  *base = st.base;
  return EMC_OK;
}

template <int N>
emc_status run_chunks(const SearchChunkArgs& proto, int n_orient, int chunk, const float2* tw,
                      NoallocResult* res, unsigned long long* best, cudaStream_t st) {
  using C = SearchCfg<N>;
  const int w = 2 * proto.radius + 1;
  for (int off = 0; off < n_orient; off += chunk) {
    SearchChunkArgs a = proto;
    a.items = proto.items + off;
    a.n_items = std::min(chunk, n_orient - off);
    EMC_CUDA(cudaMemsetAsync(a.stats, 0, sizeof(EvalStats) * a.n_items, st));
    EMC_CUDA(cudaMemsetAsync(a.keys, 0, sizeof(unsigned long long) * a.n_items, st));
    k_search_fwd_xy<N, float><<<dim3(N / C::G, a.n_items), C::NT_A, C::SMEM_A, st>>>(a, tw);
    k_search_z_mul<N><<<dim3(C::GRID_BX, (a.n_items + C::EVALS_B - 1) / C::EVALS_B), C::NT_B, C::SMEM_B, st>>>(a, tw);
    k_search_inv_peak<N><<<dim3(w, a.n_items), C::NT_BC, C::SMEM_C, st>>>(a, tw);
    k_noalloc_decode<<<(a.n_items + 127) / 128, 128, 0, st>>>(a, N, res, best);
    EMC_LAUNCH_CHECK();
  }
  return EMC_OK;
}

}  // namespace
}  // namespace emc

extern "C" {

emc_status emc_search_plain_noalloc(const float* d_ref, const float* d_mask, int n, const float* d_spectrum,
                                    double energy, const double prior[9], const float shift[3],
                                    const double* phi_theta_psi, int n_orient, int peak_radius, int interp,
                                    float* d_cc, int* d_peak, emc_search_hit* d_best, void* stream) {
  using namespace emc;
  EMC_CHECK_ARG(d_ref && d_spectrum && prior && phi_theta_psi, "emc_search_plain_noalloc: null argument");
  EMC_CHECK_ARG(n == 64 || n == 96 || n == 128, "emc_search_plain_noalloc: box %d not supported (64, 96, 128)", n);
  EMC_CHECK_ARG(n_orient >= 1 && n_orient <= EMC_NOALLOC_MAX_ORIENT,
                "emc_search_plain_noalloc: %d orientations, the static scratch holds at most %d", n_orient,
                EMC_NOALLOC_MAX_ORIENT);
  EMC_CHECK_ARG(peak_radius >= 1 && peak_radius <= EMC_NOALLOC_MAX_RADIUS && peak_radius < n / 2,
                "emc_search_plain_noalloc: peak radius %d not in [1, %d]", peak_radius, EMC_NOALLOC_MAX_RADIUS);
  EMC_CHECK_ARG(interp >= 0 && interp <= 2, "emc_search_plain_noalloc: interp %d", interp);
  EMC_CHECK_ARG(energy > 0.0, "emc_search_plain_noalloc: energy must be > 0");
  const size_t per_eval = sizeof(float2) * (s1_eval_elems(n) + s2_plane_elems(n) * (2 * peak_radius + 1));
  const size_t avail = EMC_NOALLOC_SCRATCH_BYTES - kSpecOff;
  const int chunk = (int)std::min<size_t>(kMaxChunk, avail / per_eval);
  EMC_CHECK_ARG(chunk >= 1, "emc_search_plain_noalloc: box %d with radius %d needs %zu B of scratch per "
                "evaluation, more than the %zu B available", n, peak_radius, per_eval, avail);
  unsigned char* base = nullptr;
  cudaStream_t st = as_stream(stream);
  EMC_TRY(setup_device(&base, st));

  // one host-to-device copy of everything the kernels read besides the caller's buffers
  const size_t hdr = kHdrOff, dm = kDmatOff, it = kItemOff;
  std::vector<unsigned char> host(kResOff - hdr, 0);
  DevParticle pt;
  memset(&pt, 0, sizeof(pt));
  pt.spec = reinterpret_cast<const float2*>(d_spectrum);
  pt.energy = energy;
  memcpy(pt.prior, prior, sizeof(pt.prior));
  for (int i = 0; i < 3; ++i) pt.shift[i] = shift ? shift[i] : 0.f;
  pt.ref = 0;
  pt.box = n;
  pt.orient_begin = 0;
  pt.eval_base = 0;
  DevRef rf{d_ref, d_mask, nullptr, n, EMC_DTYPE_F32};
  memcpy(host.data(), &pt, sizeof(pt));
  memcpy(host.data() + 256, &rf, sizeof(rf));
  double* dmat = reinterpret_cast<double*>(host.data() + (dm - hdr));
  EvalItem* items = reinterpret_cast<EvalItem*>(host.data() + (it - hdr));
  for (int o = 0; o < n_orient; ++o) {
    const double ang[3] = {phi_theta_psi[3 * o], phi_theta_psi[3 * o + 1],
                           phi_theta_psi[3 * o + 2] - phi_theta_psi[3 * o]};
    EMC_TRY(emc_define_matrix(ang, 1, dmat + 9 * o));
    items[o] = {0, o};
  }
  const size_t used = (it - hdr) + sizeof(EvalItem) * n_orient;
  EMC_CUDA(cudaMemcpyAsync(base + hdr, host.data(), used, cudaMemcpyHostToDevice, st));

  unsigned long long* best = reinterpret_cast<unsigned long long*>(base + kBestOff);
  unsigned* status = reinterpret_cast<unsigned*>(base + kBestOff + 8);
  EMC_CUDA(cudaMemsetAsync(best, 0, 16, st));  // best key and status word
  SearchChunkArgs a;
  a.items = reinterpret_cast<const EvalItem*>(base + it);
  a.parts = reinterpret_cast<const DevParticle*>(base + hdr);
  a.refs = reinterpret_cast<const DevRef*>(base + hdr + 256);
  a.dmat = reinterpret_cast<const double*>(base + dm);
  a.stats = reinterpret_cast<EvalStats*>(base + kStatOff);
  a.keys = reinterpret_cast<unsigned long long*>(base + kStatOff + sizeof(EvalStats) * kMaxChunk);
  a.s1 = reinterpret_cast<float2*>(base + kSpecOff);
  a.s2 = a.s1 + (size_t)chunk * s1_eval_elems(n);
  a.n_items = 0;
  a.radius = peak_radius;
  a.interp = interp;
  a.status = status;
  const float2* tw = reinterpret_cast<const float2*>(base + kTwOff) + tw_offset(n);
  NoallocResult* res = reinterpret_cast<NoallocResult*>(base + kResOff);
  emc_status rs = n == 64 ? run_chunks<64>(a, n_orient, chunk, tw, res, best, st)
                : n == 96 ? run_chunks<96>(a, n_orient, chunk, tw, res, best, st)
                          : run_chunks<128>(a, n_orient, chunk, tw, res, best, st);
  EMC_TRY(rs);
  k_noalloc_outputs<<<(n_orient + 127) / 128, 128, 0, st>>>(res, n_orient, best, d_cc, d_peak, d_best);
  EMC_LAUNCH_CHECK();
  // the host staging vector must stay alive until the copy has been consumed
  EMC_CUDA(cudaStreamSynchronize(st));
  unsigned waited_out = 0;
  EMC_CUDA(cudaMemcpy(&waited_out, status, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (waited_out) {
    set_error("emc_search_plain_noalloc: a device-side wait for bulk copies gave up; results are invalid");
    return EMC_E_TIMEOUT;
  }
  return EMC_OK;
}

}  // extern "C"
