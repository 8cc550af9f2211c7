// mrc.cu -- MRC volume I/O, tilt-table parsing and particle-window extraction: the data formats
// on either side of the alignment / averaging path.
//
// References: @MRCImage/private/readHeader.m:1-176 (header words, byte-swap detection, data
// offset 1024 + extended bytes), @MRCImage/getVolume.m:150-298 (sub-box reads, modes 0 / 1 / 2 / 6
// converted to single, mode 0 read as int8), @MRCImage/SAVE_IMG.m + private/writeHeader.m (float32
// files with min / max / mean / rms in the header, cell = n * pixel size), logicals/
// BH_isWindowValid.m (window bounds, zero padding, fractional shift) and BH_padZeros3d with the
// window extraction of transformations/BH_average3d.m:1304-1341.
//
// The device read streams z-sections through two pinned staging buffers: while section block k is
// copied to the GPU and converted to float there, block k+1 is read from the file.
#include <errno.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "common.cuh"

namespace emc {

namespace {

constexpr int kImodStamp = 1146047817;  // "IMOD"

uint32_t bswap32(uint32_t v) { return (v >> 24) | ((v >> 8) & 0xff00u) | ((v << 8) & 0xff0000u) | (v << 24); }
uint16_t bswap16(uint16_t v) { return (uint16_t)((v >> 8) | (v << 8)); }

int mode_bytes(int mode) {
  switch (mode) {
    case 0: return 1;
    case 1: return 2;
    case 2: return 4;
    case 6: return 2;
    default: return 0;
  }
}

struct Header {
  emc_mrc_header h;
  bool swap;
};

emc_status read_header(FILE* f, const char* path, Header* out) {
  unsigned char raw[1024];
  if (fseek(f, 0, SEEK_SET) != 0 || fread(raw, 1, 1024, f) != 1024) {
    set_error("mrc: %s: cannot read the 1024-byte header", path);
    return EMC_E_ARG;
  }
  auto i32 = [&](int off, bool sw) {
    uint32_t v;
    memcpy(&v, raw + off, 4);
    if (sw) v = bswap32(v);
    int32_t r;
    memcpy(&r, &v, 4);
    return r;
  };
  auto f32 = [&](int off, bool sw) {
    uint32_t v;
    memcpy(&v, raw + off, 4);
    if (sw) v = bswap32(v);
    float r;
    memcpy(&r, &v, 4);
    return r;
  };
  auto i16 = [&](int off, bool sw) {
    uint16_t v;
    memcpy(&v, raw + off, 2);
    if (sw) v = bswap16(v);
    int16_t r;
    memcpy(&r, &v, 2);
    return r;
  };
  // readHeader.m:18-40: a negative or implausibly large size means the other byte order
  bool sw = false;
  {
    const int nx = i32(0, false), ny = i32(4, false), nz = i32(8, false);
    if (nx < 0 || ny < 0 || nz < 0 || (nx > 65535 && ny > 65535 && nz > 65535)) sw = true;
  }
  emc_mrc_header& h = out->h;
  memset(&h, 0, sizeof(h));
  h.nx = i32(0, sw);
  h.ny = i32(4, sw);
  h.nz = i32(8, sw);
  h.mode = i32(12, sw);
  h.mx = i32(28, sw);
  h.my = i32(32, sw);
  h.mz = i32(36, sw);
  h.cell[0] = f32(40, sw);
  h.cell[1] = f32(44, sw);
  h.cell[2] = f32(48, sw);
  h.dmin = f32(76, sw);
  h.dmax = f32(80, sw);
  h.dmean = f32(84, sw);
  h.ext_bytes = i32(92, sw);
  h.imod_stamp = i32(152, sw);
  h.imod_flags = i32(156, sw);
  h.origin[0] = f32(196, sw);
  h.origin[1] = f32(200, sw);
  h.origin[2] = f32(204, sw);
  h.rms = f32(216, sw);
  h.data_offset = 1024L + (long)h.ext_bytes;
  (void)i16;
  for (int d = 0; d < 3; ++d) {
    const int m = d == 0 ? h.mx : d == 1 ? h.my : h.mz;
    h.pixel_size[d] = m > 0 ? h.cell[d] / (float)m : 0.f;
  }
  h.byte_swapped = sw ? 1 : 0;
  out->swap = sw;
  if (h.nx <= 0 || h.ny <= 0 || h.nz <= 0 || !mode_bytes(h.mode) || h.ext_bytes < 0) {
    set_error("mrc: %s: unsupported header (size %d %d %d, mode %d; modes 0, 1, 2, 6 are read)", path, h.nx, h.ny,
              h.nz, h.mode);
    return EMC_E_UNSUPPORTED;
  }
  return EMC_OK;
}

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

// Box [lo, hi] (1-based, inclusive) of every axis; zeros select the whole axis.
emc_status resolve_box(const emc_mrc_header& h, const int* box, int lo[3], int hi[3]) {
  const int n[3] = {h.nx, h.ny, h.nz};
  for (int d = 0; d < 3; ++d) {
    lo[d] = box && box[2 * d] ? box[2 * d] : 1;
    hi[d] = box && box[2 * d + 1] ? box[2 * d + 1] : n[d];
    if (lo[d] < 1 || hi[d] > n[d] || lo[d] > hi[d]) {
      set_error("mrc: box [%d, %d] outside 1..%d on axis %d", lo[d], hi[d], n[d], d);
      return EMC_E_ARG;
    }
  }
  return EMC_OK;
}

// Reads rows [lo..hi] of sections z0..z1 of the box into dst (raw mode bytes, rows packed).
emc_status read_sections(FILE* f, const Header& H, const int lo[3], const int hi[3], int z0, int z1,
                         unsigned char* dst) {
  const emc_mrc_header& h = H.h;
  const long mb = mode_bytes(h.mode);
  const long rx = hi[0] - lo[0] + 1, ry = hi[1] - lo[1] + 1;
  const long row_bytes = rx * mb;
  for (int z = z0; z <= z1; ++z) {
    const long sec = h.data_offset + ((long)(z - 1) * h.ny * h.nx) * mb;
    if (lo[0] == 1 && hi[0] == h.nx) {
      // whole rows: one contiguous read per section
      if (fseek(f, sec + (long)(lo[1] - 1) * h.nx * mb, SEEK_SET) != 0 ||
          fread(dst, 1, (size_t)(row_bytes * ry), f) != (size_t)(row_bytes * ry)) {
        set_error("mrc: short read in section %d", z);
        return EMC_E_ARG;
      }
      dst += row_bytes * ry;
    } else {
      for (int y = lo[1]; y <= hi[1]; ++y) {
        if (fseek(f, sec + ((long)(y - 1) * h.nx + (lo[0] - 1)) * mb, SEEK_SET) != 0 ||
            fread(dst, 1, (size_t)row_bytes, f) != (size_t)row_bytes) {
          set_error("mrc: short read in section %d row %d", z, y);
          return EMC_E_ARG;
        }
        dst += row_bytes;
      }
    }
  }
  return EMC_OK;
}

template <typename T>
__device__ __forceinline__ T load_swapped(const unsigned char* p, bool sw);
template <>
__device__ __forceinline__ int8_t load_swapped<int8_t>(const unsigned char* p, bool) { return (int8_t)p[0]; }
template <>
__device__ __forceinline__ int16_t load_swapped<int16_t>(const unsigned char* p, bool sw) {
  const uint16_t v = sw ? (uint16_t)((p[0] << 8) | p[1]) : (uint16_t)(p[0] | (p[1] << 8));
  return (int16_t)v;
}
template <>
__device__ __forceinline__ uint16_t load_swapped<uint16_t>(const unsigned char* p, bool sw) {
  return sw ? (uint16_t)((p[0] << 8) | p[1]) : (uint16_t)(p[0] | (p[1] << 8));
}
template <>
__device__ __forceinline__ float load_swapped<float>(const unsigned char* p, bool sw) {
  const uint32_t v = sw ? ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]
                        : (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
  return __uint_as_float(v);
}

template <typename T>
__global__ void k_mrc_convert(const unsigned char* __restrict__ raw, long n, int swap, float* __restrict__ out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = (float)load_swapped<T>(raw + i * (long)sizeof(T), swap != 0);
}

emc_status convert_on_device(int mode, const unsigned char* d_raw, long n, bool swap, float* d_out,
                             cudaStream_t st) {
  const int blocks = (int)std::max<long>(1, std::min<long>((n + 255) / 256, 8L * device_sm_count()));
  switch (mode) {
    case 0: k_mrc_convert<int8_t><<<blocks, 256, 0, st>>>(d_raw, n, swap, d_out); break;
    case 1: k_mrc_convert<int16_t><<<blocks, 256, 0, st>>>(d_raw, n, swap, d_out); break;
    case 2: k_mrc_convert<float><<<blocks, 256, 0, st>>>(d_raw, n, swap, d_out); break;
    case 6: k_mrc_convert<uint16_t><<<blocks, 256, 0, st>>>(d_raw, n, swap, d_out); break;
    default: set_error("mrc: mode %d", mode); return EMC_E_UNSUPPORTED;
  }
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

// Host-side conversion (same rules as the device kernel).
void convert_on_host(int mode, const unsigned char* raw, long n, bool sw, float* out) {
  for (long i = 0; i < n; ++i) {
    const unsigned char* p = raw + i * mode_bytes(mode);
    switch (mode) {
      case 0: out[i] = (float)(int8_t)p[0]; break;
      case 1: {
        const uint16_t v = sw ? (uint16_t)((p[0] << 8) | p[1]) : (uint16_t)(p[0] | (p[1] << 8));
        out[i] = (float)(int16_t)v;
        break;
      }
      case 6: out[i] = (float)(sw ? (uint16_t)((p[0] << 8) | p[1]) : (uint16_t)(p[0] | (p[1] << 8))); break;
      default: {
        uint32_t v;
        memcpy(&v, p, 4);
        if (sw) v = bswap32(v);
        memcpy(out + i, &v, 4);
      }
    }
  }
}

// --------------------------------------------------------------- window extraction
struct WindowArgs {
  long vx, vy, vz;  // volume size
  int w[3];         // window size
};

// out[p][k][j][i] = vol(start + (i, j, k)) inside the volume, 0 outside (BH_isWindowValid +
// BH_padZeros3d with a zero fill).  start: 0-based volume index of window voxel 0, per window.
// One warp per window row: the row's source segment is contiguous, so loads and stores coalesce
// and no per-element index division is needed.
__global__ void __launch_bounds__(256) k_extract(const float* __restrict__ vol, WindowArgs a,
                                                 const int* __restrict__ start, float* __restrict__ out) {
  const int p = blockIdx.y;
  const int sx = start[3 * p], sy = start[3 * p + 1], sz = start[3 * p + 2];
  const long nrows = (long)a.w[1] * a.w[2];
  float* dst = out + (long)p * nrows * a.w[0];
  const int lane = threadIdx.x & 31;
  const long warp = blockIdx.x * (long)(blockDim.x >> 5) + (threadIdx.x >> 5);
  const long nwarps = (long)gridDim.x * (blockDim.x >> 5);
  // the valid x range of every row of this window
  const long x_top = a.vx - sx;
  const int x_lo = sx < 0 ? -sx : 0, x_hi = x_top < a.w[0] ? (int)x_top : a.w[0];
  // RB rows per warp and step, every load of the step issued before its stores (a 64-voxel row is
  // only two loads per lane: one row at a time left the copy latency-bound)
  constexpr int RB = 8;
  for (long row0 = warp * RB; row0 < nrows; row0 += nwarps * RB) {
    for (int i0 = 0; i0 < a.w[0]; i0 += 64) {
      float v[RB][2];
#pragma unroll
      for (int q = 0; q < RB; ++q) {
        const long row = row0 + q;
        const int j = (int)(row % a.w[1]), k = (int)(row / a.w[1]);
        const long gy = sy + j, gz = sz + k;
        const bool in_yz = row < nrows && gy >= 0 && gz >= 0 && gy < a.vy && gz < a.vz;
        const long base = (gz * a.vy + gy) * a.vx + sx;  // dereferenced only for in-volume voxels
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int i = i0 + lane + 32 * h;
          v[q][h] = (in_yz && i >= x_lo && i < x_hi) ? __ldg(vol + base + i) : 0.f;
        }
      }
#pragma unroll
      for (int q = 0; q < RB; ++q) {
        const long row = row0 + q;
        if (row >= nrows) break;
        float* d = dst + row * a.w[0];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int i = i0 + lane + 32 * h;
          if (i < a.w[0]) d[i] = v[q][h];
        }
      }
    }
  }
}

}  // namespace
}  // namespace emc

extern "C" {

emc_status emc_mrc_read_header(const char* path, emc_mrc_header* out) {
  EMC_CHECK_ARG(path && out, "emc_mrc_read_header: null argument");
  emc::File F;
  F.f = fopen(path, "rb");
  EMC_CHECK_ARG(F.f, "emc_mrc_read_header: cannot open %s (%s)", path, strerror(errno));
  emc::Header H;
  EMC_TRY(emc::read_header(F.f, path, &H));
  *out = H.h;
  return EMC_OK;
}

emc_status emc_mrc_read(const char* path, const int* box, float* h_out) {
  EMC_CHECK_ARG(path && h_out, "emc_mrc_read: null argument");
  emc::File F;
  F.f = fopen(path, "rb");
  EMC_CHECK_ARG(F.f, "emc_mrc_read: cannot open %s (%s)", path, strerror(errno));
  emc::Header H;
  EMC_TRY(emc::read_header(F.f, path, &H));
  int lo[3], hi[3];
  EMC_TRY(emc::resolve_box(H.h, box, lo, hi));
  const long rx = hi[0] - lo[0] + 1, ry = hi[1] - lo[1] + 1;
  const long mb = emc::mode_bytes(H.h.mode);
  std::vector<unsigned char> raw((size_t)(rx * ry * mb));
  for (int z = lo[2]; z <= hi[2]; ++z) {
    EMC_TRY(emc::read_sections(F.f, H, lo, hi, z, z, raw.data()));
    emc::convert_on_host(H.h.mode, raw.data(), rx * ry, H.swap, h_out + (long)(z - lo[2]) * rx * ry);
  }
  return EMC_OK;
}

emc_status emc_mrc_read_device(const char* path, const int* box, float* d_out, void* stream) {
  EMC_CHECK_ARG(path && d_out, "emc_mrc_read_device: null argument");
  emc::File F;
  F.f = fopen(path, "rb");
  EMC_CHECK_ARG(F.f, "emc_mrc_read_device: cannot open %s (%s)", path, strerror(errno));
  emc::Header H;
  EMC_TRY(emc::read_header(F.f, path, &H));
  int lo[3], hi[3];
  EMC_TRY(emc::resolve_box(H.h, box, lo, hi));
  cudaStream_t st = emc::as_stream(stream);
  const long rx = hi[0] - lo[0] + 1, ry = hi[1] - lo[1] + 1, nsec = hi[2] - lo[2] + 1;
  const long mb = emc::mode_bytes(H.h.mode);
  const long sec_bytes = rx * ry * mb;
  // blocks of sections of about 32 MB, double-buffered
  const long per = std::max<long>(1, std::min<long>(nsec, (32L << 20) / std::max<long>(1, sec_bytes)));
  const size_t buf_bytes = (size_t)(per * sec_bytes);
  unsigned char* pinned[2] = {nullptr, nullptr};
  unsigned char* d_raw[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  emc_status rs = EMC_OK;
  for (int b = 0; b < 2 && rs == EMC_OK; ++b) {
    if (cudaMallocHost((void**)&pinned[b], buf_bytes) != cudaSuccess ||
        cudaMalloc((void**)&d_raw[b], buf_bytes) != cudaSuccess ||
        cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming) != cudaSuccess) {
      emc::set_error("emc_mrc_read_device: staging allocation of %zu bytes failed", buf_bytes);
      rs = EMC_E_OOM;
    }
  }
  bool pending[2] = {false, false};
  for (long s0 = 0, k = 0; s0 < nsec && rs == EMC_OK; s0 += per, ++k) {
    const int b = (int)(k & 1);
    const long cnt = std::min(per, nsec - s0);
    // the copy that last used this staging buffer must be finished before it is refilled
    if (pending[b] && cudaEventSynchronize(done[b]) != cudaSuccess) {
      rs = EMC_E_CUDA;
      break;
    }
    rs = emc::read_sections(F.f, H, lo, hi, lo[2] + (int)s0, lo[2] + (int)(s0 + cnt - 1), pinned[b]);
    if (rs != EMC_OK) break;
    if (cudaMemcpyAsync(d_raw[b], pinned[b], (size_t)(cnt * sec_bytes), cudaMemcpyHostToDevice, st) != cudaSuccess) {
      rs = EMC_E_CUDA;
      break;
    }
    rs = emc::convert_on_device(H.h.mode, d_raw[b], cnt * rx * ry, H.swap, d_out + s0 * rx * ry, st);
    if (rs != EMC_OK) break;
    if (cudaEventRecord(done[b], st) != cudaSuccess) {
      rs = EMC_E_CUDA;
      break;
    }
    pending[b] = true;
  }
  if (rs == EMC_E_CUDA) emc::set_error("emc_mrc_read_device: %s", cudaGetErrorString(cudaGetLastError()));
  // device buffers are released only after the queued copies and conversions are done
  if (cudaStreamSynchronize(st) != cudaSuccess && rs == EMC_OK) {
    emc::set_error("emc_mrc_read_device: %s", cudaGetErrorString(cudaGetLastError()));
    rs = EMC_E_CUDA;
  }
  for (int b = 0; b < 2; ++b) {
    if (pinned[b]) cudaFreeHost(pinned[b]);
    if (d_raw[b]) cudaFree(d_raw[b]);
    if (done[b]) cudaEventDestroy(done[b]);
  }
  return rs;
}

emc_status emc_mrc_write(const char* path, const float* h_vol, int nx, int ny, int nz, const float pixel_size[3],
                         const float origin[3]) {
  EMC_CHECK_ARG(path && h_vol && nx > 0 && ny > 0 && nz > 0, "emc_mrc_write: bad argument");
  // header statistics as SAVE_IMG computes them: min, max, mean and std(std(std(vol))) (n - 1)
  const long n = (long)nx * ny * nz;
  float mn = h_vol[0], mx = h_vol[0];
  double sum = 0.0;
  for (long i = 0; i < n; ++i) {
    mn = std::min(mn, h_vol[i]);
    mx = std::max(mx, h_vol[i]);
    sum += h_vol[i];
  }
  auto stdv = [](const std::vector<double>& v) {
    if (v.size() < 2) return 0.0;
    double m = 0.0;
    for (double x : v) m += x;
    m /= (double)v.size();
    double s = 0.0;
    for (double x : v) s += (x - m) * (x - m);
    return sqrt(s / (double)(v.size() - 1));
  };
  std::vector<double> s1((size_t)ny * nz);
  {
    std::vector<double> row(nx);
    for (long yz = 0; yz < (long)ny * nz; ++yz) {
      for (int x = 0; x < nx; ++x) row[x] = h_vol[yz * nx + x];
      s1[yz] = stdv(row);
    }
  }
  std::vector<double> s2(nz);
  {
    std::vector<double> col(ny);
    for (int z = 0; z < nz; ++z) {
      for (int y = 0; y < ny; ++y) col[y] = s1[(size_t)z * ny + y];
      s2[z] = stdv(col);
    }
  }
  // std of a size-1 dimension is 0 along that dimension; MATLAB's std walks the first
  // non-singleton dimension, which the nested loops above follow for nx, ny, nz > 1
  const double rms = nx > 1 && ny > 1 && nz > 1 ? stdv(s2) : 0.0;
  unsigned char hdr[1024];
  memset(hdr, 0, sizeof(hdr));
  auto put_i = [&](int off, int32_t v) { memcpy(hdr + off, &v, 4); };
  auto put_f = [&](int off, float v) { memcpy(hdr + off, &v, 4); };
  put_i(0, nx);
  put_i(4, ny);
  put_i(8, nz);
  put_i(12, 2);
  put_i(28, nx);
  put_i(32, ny);
  put_i(36, nz);
  const float px[3] = {pixel_size ? pixel_size[0] : 1.f, pixel_size ? pixel_size[1] : 1.f,
                       pixel_size ? pixel_size[2] : 1.f};
  put_f(40, nx * px[0]);
  put_f(44, ny * px[1]);
  put_f(48, nz * px[2]);
  put_f(52, 90.f);
  put_f(56, 90.f);
  put_f(60, 90.f);
  put_i(64, 1);
  put_i(68, 2);
  put_i(72, 3);
  put_f(76, mn);
  put_f(80, mx);
  put_f(84, (float)(sum / (double)n));
  put_i(88, 1);  // space group
  put_i(92, 0);  // no extended header
  if (origin) {
    put_f(196, origin[0]);
    put_f(200, origin[1]);
    put_f(204, origin[2]);
  }
  memcpy(hdr + 208, "MAP ", 4);
  hdr[212] = 0x44;  // little-endian machine stamp
  hdr[213] = 0x44;
  put_f(216, (float)rms);
  FILE* f = fopen(path, "wb");
  EMC_CHECK_ARG(f, "emc_mrc_write: cannot create %s (%s)", path, strerror(errno));
  const bool ok = fwrite(hdr, 1, 1024, f) == 1024 && fwrite(h_vol, sizeof(float), (size_t)n, f) == (size_t)n;
  const bool closed = fclose(f) == 0;
  EMC_CHECK_ARG(ok && closed, "emc_mrc_write: write to %s failed", path);
  return EMC_OK;
}

emc_status emc_tlt_read(const char* path, double* out, int max_rows, int* rows, int* cols) {
  EMC_CHECK_ARG(path && rows && cols, "emc_tlt_read: null argument");
  FILE* f = fopen(path, "r");
  EMC_CHECK_ARG(f, "emc_tlt_read: cannot open %s (%s)", path, strerror(errno));
  std::vector<std::vector<double>> table;
  char line[8192];
  int ncol = -1;
  emc_status rs = EMC_OK;
  while (fgets(line, sizeof(line), f)) {
    std::vector<double> r;
    char* p = line;
    while (true) {
      while (*p == ' ' || *p == '\t' || *p == ',') ++p;
      if (*p == '\0' || *p == '\n' || *p == '\r' || *p == '%' || *p == '#') break;
      char* end = nullptr;
      const double v = strtod(p, &end);
      if (end == p) {
        emc::set_error("emc_tlt_read: %s: not a number near '%.16s'", path, p);
        rs = EMC_E_ARG;
        break;
      }
      r.push_back(v);
      p = end;
    }
    if (rs != EMC_OK) break;
    if (r.empty()) continue;
    if (ncol < 0) ncol = (int)r.size();
    if ((int)r.size() != ncol) {
      emc::set_error("emc_tlt_read: %s: row %zu has %zu columns, expected %d", path, table.size() + 1, r.size(), ncol);
      rs = EMC_E_ARG;
      break;
    }
    table.push_back(std::move(r));
  }
  fclose(f);
  if (rs != EMC_OK) return rs;
  *rows = (int)table.size();
  *cols = ncol < 0 ? 0 : ncol;
  if (out) {
    EMC_CHECK_ARG(max_rows >= (int)table.size(), "emc_tlt_read: %d rows do not fit in %d", (int)table.size(),
                  max_rows);
    // row-major: out[r * cols + c]
    for (size_t r = 0; r < table.size(); ++r)
      for (int c = 0; c < ncol; ++c) out[r * ncol + c] = table[r][c];
  }
  return EMC_OK;
}

emc_status emc_window_bounds(const int volume_size[3], const int window_size[3], double mask_radius,
                             const double center[3], int start[3], int pad_low[3], int pad_top[3],
                             double shift[3], int* valid) {
  EMC_CHECK_ARG(volume_size && window_size && center && valid, "emc_window_bounds: null argument");
  // BH_isWindowValid.m: 1-based window [winCenter - winLow, winCenter + winTop]
  const double min_size = (mask_radius + 6.0) * 2.0;
  int ok = 1;
  for (int d = 0; d < 3; ++d) {
    const int W = window_size[d];
    const int win_low = (int)ceil((W - 1) / 2.0);
    const int win_top = win_low - ((W - 1) % 2);
    const double c = floor(center[d]);
    const double low = c - win_low;
    const double top = volume_size[d] - (c + win_top);
    const int pl = low <= 0 ? (int)(fabs(low) + 1) : 0;
    const int pt = top <= 0 ? (int)fabs(top) : 0;
    if (start) start[d] = (int)low - 1;  // 0-based volume index of window voxel 0
    if (pad_low) pad_low[d] = pl;
    if (pad_top) pad_top[d] = pt;
    if (shift) shift[d] = center[d] - c;
    if (W - pl - pt - min_size < -2) ok = 0;
  }
  *valid = ok;
  return EMC_OK;
}

emc_status emc_extract_windows(const float* d_vol, int nx, int ny, int nz, const int window_size[3],
                               const double* centers, int count, double mask_radius, float* d_out,
                               double* shifts, int* valid, void* stream) {
  EMC_CHECK_ARG(d_vol && window_size && centers && d_out && count >= 0, "emc_extract_windows: bad argument");
  EMC_CHECK_ARG(nx > 0 && ny > 0 && nz > 0 && window_size[0] > 0 && window_size[1] > 0 && window_size[2] > 0,
                "emc_extract_windows: bad size");
  if (count == 0) return EMC_OK;
  const int vs[3] = {nx, ny, nz};
  std::vector<int> start(3 * (size_t)count);
  for (int p = 0; p < count; ++p) {
    int ok = 0;
    EMC_TRY(emc_window_bounds(vs, window_size, mask_radius, centers + 3 * (size_t)p, start.data() + 3 * (size_t)p,
                              nullptr, nullptr, shifts ? shifts + 3 * (size_t)p : nullptr, &ok));
    if (valid) valid[p] = ok;
  }
  cudaStream_t st = emc::as_stream(stream);
  int* d_start = nullptr;
  EMC_CUDA(cudaMallocAsync((void**)&d_start, sizeof(int) * start.size(), st));
  emc_status rs = EMC_OK;
  if (cudaMemcpyAsync(d_start, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice, st) != cudaSuccess) {
    rs = EMC_E_CUDA;
  } else {
    emc::WindowArgs a;
    a.vx = nx;
    a.vy = ny;
    a.vz = nz;
    for (int d = 0; d < 3; ++d) a.w[d] = window_size[d];
    const long nw = (long)window_size[0] * window_size[1] * window_size[2];
    const long nrows = (long)window_size[1] * window_size[2];
    const int gx = (int)std::max<long>(1, std::min<long>((nrows + 63) / 64, 64));  // 8 warps x 8 rows per block
    for (int p0 = 0; p0 < count && rs == EMC_OK; p0 += 65535) {
      const int cnt = std::min(65535, count - p0);
      emc::k_extract<<<dim3(gx, cnt), 256, 0, st>>>(d_vol, a, d_start + 3 * (size_t)p0, d_out + (size_t)p0 * nw);
      if (cudaGetLastError() != cudaSuccess) rs = EMC_E_CUDA;
    }
  }
  if (rs == EMC_E_CUDA) emc::set_error("emc_extract_windows: %s", cudaGetErrorString(cudaGetLastError()));
  cudaFreeAsync(d_start, st);
  // the host start vector is read by the async copy: wait before it goes out of scope
  if (cudaStreamSynchronize(st) != cudaSuccess && rs == EMC_OK) rs = EMC_E_CUDA;
  return rs;
}

}  // extern "C"
