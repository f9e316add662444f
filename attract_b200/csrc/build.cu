// Receptor-side kernels: potential grid builder (K3), neighbour-grid builder
// (K4: count -> scan -> fill) and the dense-grid -> brick repack (K5).
#include <math.h>

#include "common.cuh"

namespace att {

// ---------------------------------------------------------------------------
// K3: energy + force voxels (test-calc-grid-energy.py:154-196, with forces)
// ---------------------------------------------------------------------------
constexpr int BUILD_THREADS = 256;

__global__ void __launch_bounds__(BUILD_THREADS)
build_potential_kernel(AttGridGeom g, const float4* __restrict__ rec, int n_rec, const float4* __restrict__ pair,
                       int n_rtypes, float cutoff2, int outer, float* __restrict__ out) {
  __shared__ float4 srec[BUILD_THREADS];
  const int lt = blockIdx.y;
  const int nx = outer ? g.dim2[0] : g.dim[0];
  const int ny = outer ? g.dim2[1] : g.dim[1];
  const int nz = outer ? g.dim2[2] : g.dim[2];
  const long long npts = (long long)nx * ny * nz;
  const long long pt = (long long)blockIdx.x * BUILD_THREADS + threadIdx.x;
  const bool live = pt < npts;
  const int iz = (int)(pt % nz);
  const int iy = (int)((pt / nz) % ny);
  const int ix = (int)(pt / ((long long)nz * ny));
  float px, py, pz;
  if (!outer) {
    px = g.origin[0] + ix * g.spacing;
    py = g.origin[1] + iy * g.spacing;
    pz = g.origin[2] + iz * g.spacing;
  } else {
    px = g.origin[0] + (2.f * ix - g.extension) * g.spacing;
    py = g.origin[1] + (2.f * iy - g.extension) * g.spacing;
    pz = g.origin[2] + (2.f * iz - g.extension) * g.spacing;
  }
  const double p = g.plateau;
  const double p2 = p * p;
  double e = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
  const float4* prow = pair + (long long)lt * n_rtypes * 2;
  for (int base = 0; base < n_rec; base += BUILD_THREADS) {
    __syncthreads();
    if (base + threadIdx.x < n_rec) srec[threadIdx.x] = rec[base + threadIdx.x];
    __syncthreads();
    const int m = min(BUILD_THREADS, n_rec - base);
    if (!live) continue;
    for (int k = 0; k < m; ++k) {
      const float4 r = srec[k];
      const double dx = (double)px - r.x, dy = (double)py - r.y, dz = (double)pz - r.z;
      const double dsq = dx * dx + dy * dy + dz * dz;
      if (!(dsq < cutoff2)) continue;
      const int rt = __float_as_int(r.w);
      if ((unsigned)rt >= (unsigned)n_rtypes) continue;
      const float4 q0 = prow[rt * 2], q1 = prow[rt * 2 + 1];  // rc ac emin rmin2 | ivor eplat gplat rcap2
      double scale;
      if (dsq < p2) {
        e += q1.y;
        scale = dsq > 0.0 ? (double)q1.z * p / sqrt(dsq) : 0.0;
      } else {
        const double d2 = fmax(dsq, (double)q1.w);
        const double rr2 = 1.0 / d2;
        const double rr6 = rr2 * rr2 * rr2;
        const double vlj = ((double)q0.x * rr2 - q0.y) * rr6;
        const bool near = d2 < q0.w;
        e += near ? vlj + ((double)q1.x - 1.0) * q0.z : (double)q1.x * vlj;
        const double dv = rr6 * rr2 * (3.0 * q0.y - 4.0 * q0.x * rr2);
        scale = (dsq < q1.w) ? 0.0 : (near ? dv : q1.x * dv);
      }
      fx -= 2.0 * scale * dx;
      fy -= 2.0 * scale * dy;
      fz -= 2.0 * scale * dz;
    }
  }
  if (live) {
    float4 v = make_float4((float)e, (float)fx, (float)fy, (float)fz);
    reinterpret_cast<float4*>(out)[(long long)lt * npts + pt] = v;
  }
}

cudaError_t launch_build_potential(const AttGridGeom& g, const float* rec, int n_rec, const float* pair,
                                   int n_rtypes, int n_ltypes, float cutoff, int outer, float* out,
                                   cudaStream_t st) {
  const long long npts = outer ? (long long)g.dim2[0] * g.dim2[1] * g.dim2[2]
                               : (long long)g.dim[0] * g.dim[1] * g.dim[2];
  dim3 grid((unsigned)((npts + BUILD_THREADS - 1) / BUILD_THREADS), (unsigned)n_ltypes);
  build_potential_kernel<<<grid, BUILD_THREADS, 0, st>>>(g, reinterpret_cast<const float4*>(rec), n_rec,
                                                         reinterpret_cast<const float4*>(pair), n_rtypes,
                                                         cutoff * cutoff, outer, out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// K4: neighbour lists (test-calc-grid-energy.py:90-103) as CSR
// ---------------------------------------------------------------------------
constexpr int SCAN_THREADS = 1024;

// Grid point and squared distance with every operation rounded on its own
// (no contraction into FMA): the list membership test d^2 <= r^2 is then a
// fixed float32 computation that a host restatement reproduces bit for bit.
__device__ __forceinline__ void point_of(const AttGridGeom& g, long long v, float& x, float& y, float& z) {
  const int nz = g.dim[2], ny = g.dim[1];
  const int iz = (int)(v % nz);
  const int iy = (int)((v / nz) % ny);
  const int ix = (int)(v / ((long long)nz * ny));
  x = __fadd_rn(g.origin[0], __fmul_rn((float)ix, g.spacing));
  y = __fadd_rn(g.origin[1], __fmul_rn((float)iy, g.spacing));
  z = __fadd_rn(g.origin[2], __fmul_rn((float)iz, g.spacing));
}

__device__ __forceinline__ float dist2_rn(float x, float y, float z, const float4& r) {
  const float dx = __fsub_rn(x, r.x), dy = __fsub_rn(y, r.y), dz = __fsub_rn(z, r.z);
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// count + block-local exclusive scan; block totals to ws
__global__ void __launch_bounds__(SCAN_THREADS)
nb_count_kernel(AttGridGeom g, const float4* __restrict__ rec, int n_rec, float r2, uint2* __restrict__ hdr,
                unsigned* __restrict__ ws, long long nvox) {
  __shared__ float4 srec[SCAN_THREADS];
  __shared__ unsigned wsum[SCAN_THREADS / 32];
  const long long v = (long long)blockIdx.x * SCAN_THREADS + threadIdx.x;
  float x = 0.f, y = 0.f, z = 0.f;
  if (v < nvox) point_of(g, v, x, y, z);
  unsigned c = 0;
  for (int base = 0; base < n_rec; base += SCAN_THREADS) {
    __syncthreads();
    if (base + threadIdx.x < n_rec) srec[threadIdx.x] = rec[base + threadIdx.x];
    __syncthreads();
    const int m = min(SCAN_THREADS, n_rec - base);
    for (int k = 0; k < m; ++k) {
      c += dist2_rn(x, y, z, srec[k]) <= r2;
    }
  }
  if (v >= nvox) c = 0;
  // block exclusive scan
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned inc = c;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const unsigned t = __shfl_up_sync(0xffffffffu, inc, off);
    if (lane >= off) inc += t;
  }
  if (lane == 31) wsum[w] = inc;
  __syncthreads();
  if (w == 0) {
    unsigned s = wsum[lane];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const unsigned t = __shfl_up_sync(0xffffffffu, s, off);
      if (lane >= off) s += t;
    }
    wsum[lane] = s;  // inclusive per warp
  }
  __syncthreads();
  const unsigned before = (w > 0 ? wsum[w - 1] : 0u) + inc - c;
  if (v < nvox) hdr[v] = make_uint2(before, c);
  if (threadIdx.x == SCAN_THREADS - 1) ws[blockIdx.x] = wsum[SCAN_THREADS / 32 - 1];
}

// exclusive scan of the block totals (one block, sequential chunks)
__global__ void __launch_bounds__(SCAN_THREADS)
nb_scan_blocks_kernel(unsigned* __restrict__ ws, int nblk, unsigned long long* __restrict__ total) {
  __shared__ unsigned wsum[SCAN_THREADS / 32];
  __shared__ unsigned long long carry;
  if (threadIdx.x == 0) carry = 0ull;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int base = 0; base < nblk; base += SCAN_THREADS) {
    const int i = base + threadIdx.x;
    const unsigned c = i < nblk ? ws[i] : 0u;
    unsigned inc = c;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const unsigned t = __shfl_up_sync(0xffffffffu, inc, off);
      if (lane >= off) inc += t;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
      unsigned s = wsum[lane];
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, s, off);
        if (lane >= off) s += t;
      }
      wsum[lane] = s;
    }
    __syncthreads();
    const unsigned long long cb = carry;
    if (i < nblk) ws[i] = (unsigned)(cb + (w > 0 ? wsum[w - 1] : 0u) + inc - c);
    __syncthreads();
    if (threadIdx.x == 0) carry = cb + wsum[SCAN_THREADS / 32 - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void nb_add_kernel(uint2* __restrict__ hdr, const unsigned* __restrict__ ws, long long nvox) {
  const long long v = (long long)blockIdx.x * SCAN_THREADS + threadIdx.x;
  if (v < nvox) hdr[v].x += ws[blockIdx.x];
}

__global__ void __launch_bounds__(256)
nb_fill_kernel(AttGridGeom g, const float4* __restrict__ rec, int n_rec, float r2, const uint2* __restrict__ hdr,
               uint16_t* __restrict__ list, long long nvox) {
  __shared__ float4 srec[256];
  const long long v = (long long)blockIdx.x * 256 + threadIdx.x;
  float x = 0.f, y = 0.f, z = 0.f;
  uint2 h = make_uint2(0u, 0u);
  if (v < nvox) {
    point_of(g, v, x, y, z);
    h = hdr[v];
  }
  unsigned pos = 0;
  for (int base = 0; base < n_rec; base += 256) {
    __syncthreads();
    if (base + threadIdx.x < n_rec) srec[threadIdx.x] = rec[base + threadIdx.x];
    __syncthreads();
    const int m = min(256, n_rec - base);
    if (v >= nvox) continue;
    for (int k = 0; k < m; ++k) {
      if (dist2_rn(x, y, z, srec[k]) <= r2 && pos < h.y) list[h.x + pos++] = (uint16_t)(base + k);
    }
  }
}

long long nb_workspace_bytes(long long nvox) {
  return ((nvox + SCAN_THREADS - 1) / SCAN_THREADS) * (long long)sizeof(unsigned) + 256;
}

cudaError_t launch_nb_count(const AttGridGeom& g, const float* rec, int n_rec, float radius, uint32_t* hdr,
                            unsigned long long* total, void* ws, cudaStream_t st) {
  const long long nvox = (long long)g.dim[0] * g.dim[1] * g.dim[2];
  const int nblk = (int)((nvox + SCAN_THREADS - 1) / SCAN_THREADS);
  unsigned* w = reinterpret_cast<unsigned*>(ws);
  nb_count_kernel<<<nblk, SCAN_THREADS, 0, st>>>(g, reinterpret_cast<const float4*>(rec), n_rec, radius * radius,
                                                 reinterpret_cast<uint2*>(hdr), w, nvox);
  nb_scan_blocks_kernel<<<1, SCAN_THREADS, 0, st>>>(w, nblk, total);
  nb_add_kernel<<<nblk, SCAN_THREADS, 0, st>>>(reinterpret_cast<uint2*>(hdr), w, nvox);
  return cudaGetLastError();
}

cudaError_t launch_nb_fill(const AttGridGeom& g, const float* rec, int n_rec, float radius, const uint32_t* hdr,
                           uint16_t* list, cudaStream_t st) {
  const long long nvox = (long long)g.dim[0] * g.dim[1] * g.dim[2];
  nb_fill_kernel<<<(unsigned)((nvox + 255) / 256), 256, 0, st>>>(g, reinterpret_cast<const float4*>(rec), n_rec,
                                                                  radius * radius,
                                                                  reinterpret_cast<const uint2*>(hdr), list, nvox);
  return cudaGetLastError();
}

// CSR -> fixed-size records {inline entries, u16 count, u32 overflow index}:
// the entries start the record, so that a reader takes four at a time in
// 8-byte loads
__global__ void nb_pack_kernel(const uint2* __restrict__ hdr, const uint16_t* __restrict__ list, long long nvox,
                               int rec_bytes, unsigned char* __restrict__ out) {
  const int inl = ATT_NB_INLINE(rec_bytes);
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
       v += (long long)gridDim.x * blockDim.x) {
    const uint2 h = hdr[v];
    unsigned char* r = out + v * rec_bytes;
    uint16_t* e = reinterpret_cast<uint16_t*>(r);
    for (int i = 0; i < inl; ++i) e[i] = (i < (int)h.y) ? list[h.x + i] : (uint16_t)ATT_NB_EMPTY;
    *reinterpret_cast<uint16_t*>(r + rec_bytes - 6) = (uint16_t)min(h.y, 65535u);
    *reinterpret_cast<unsigned*>(r + rec_bytes - 4) = h.x + (unsigned)inl;
  }
}

cudaError_t launch_nb_pack(const uint32_t* hdr, const uint16_t* list, long long nvox, int rec_bytes, void* out,
                           cudaStream_t st) {
  nb_pack_kernel<<<148 * 8, 256, 0, st>>>(reinterpret_cast<const uint2*>(hdr), list, nvox, rec_bytes,
                                          reinterpret_cast<unsigned char*>(out));
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// K5: dense [T][X][Y][Z][4] -> bricks [T][inner+outer][8 corners]
// ---------------------------------------------------------------------------
__global__ void repack_kernel(const float4* __restrict__ src, int T, int dx, int dy, int dz, long long brick0,
                              long long type_stride, float4* __restrict__ dst) {
  const long long nb = (long long)(dx - 1) * (dy - 1) * (dz - 1);
  const long long total = (long long)T * nb * 8;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i & 7);
    const long long bi = i >> 3;
    const int t = (int)(bi / nb);
    const long long b = bi - (long long)t * nb;
    const int iz = (int)(b % (dz - 1));
    const int iy = (int)((b / (dz - 1)) % (dy - 1));
    const int ix = (int)(b / ((long long)(dz - 1) * (dy - 1)));
    const int x = ix + ((c >> 2) & 1), y = iy + ((c >> 1) & 1), z = iz + (c & 1);
    dst[((long long)t * type_stride + brick0 + b) * 8 + c] = src[(((long long)t * dx + x) * dy + y) * dz + z];
  }
}

cudaError_t launch_repack(const AttGridGeom& g, const float* inner, const float* outer, void* bricks,
                          cudaStream_t st) {
  const long long ni = (long long)(g.dim[0] - 1) * (g.dim[1] - 1) * (g.dim[2] - 1);
  const long long no = outer ? (long long)(g.dim2[0] - 1) * (g.dim2[1] - 1) * (g.dim2[2] - 1) : 0;
  const long long stride = ni + no;
  float4* dst = reinterpret_cast<float4*>(bricks);
  repack_kernel<<<148 * 8, 256, 0, st>>>(reinterpret_cast<const float4*>(inner), g.n_types, g.dim[0], g.dim[1],
                                         g.dim[2], 0, stride, dst);
  if (outer) {
    repack_kernel<<<148 * 8, 256, 0, st>>>(reinterpret_cast<const float4*>(outer), g.n_types, g.dim2[0],
                                           g.dim2[1], g.dim2[2], ni, stride, dst);
  }
  return cudaGetLastError();
}

}  // namespace att

// ---------------------------------------------------------------------------
// att_nbgrid_count_noalloc: the neighbour-list count + scan of
// att_nbgrid_count with its scan workspace (one word per 1024 grid points) in
// a fixed device array of this library instead of caller memory, for callers
// that cannot allocate device memory themselves.
// ---------------------------------------------------------------------------
#include <mutex>
#include <stdio.h>

namespace att {
int report_error(int code, const char* msg);
int check_geom(const AttGridGeom* g);  // the validation of att_nbgrid_count (capi.cu)
}

// Fixed scan workspace: 8192 words = 32 KB, i.e. grids of up to 8192 * 1024
// inner points.  Every device that loads the library holds it until exit.
static __device__ __align__(256) unsigned g_nbgrid_scan_ws[ATT_NBGRID_NOALLOC_MAX_VOXELS / 1024];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scan_ws_mutex;
struct ScanWsEntry {
  void* ctx;   // the CUDA context the address belongs to
  void* addr;  // device address of g_nbgrid_scan_ws in that context
};
ScanWsEntry g_scan_ws[kMaxDevices] = {};

// cuCtxGetCurrent through the runtime's driver entry point (no link-time
// dependency on the driver library); NULL when unavailable.
typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(f);
  }();
  return fn;
}

// Device address of the fixed workspace on the current device.  The name
// g_nbgrid_scan_ws in host code is only a host-side stand-in for the symbol;
// the kernel must be given the address that cudaGetSymbolAddress returns with
// that device current.  Looked up on the first call on a device and cached per
// device together with the context it was taken in: after a device reset (or
// with another context current) the stale address is dropped and looked up
// again.  Without a current context handle (none made current yet, or no
// driver entry point) the address is looked up on every call.
int scan_ws_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return att::report_error(ATT_E_CUDA, "att_nbgrid_count_noalloc: cudaGetDevice failed");
  if (dev < 0 || dev >= kMaxDevices)
    return att::report_error(ATT_E_UNSUPPORTED, "att_nbgrid_count_noalloc: device index beyond 64");
  void* ctx = nullptr;
  CtxGetCurrentFn get = ctx_get_current();
  const bool have_ctx = get != nullptr && get(&ctx) == 0 && ctx != nullptr;
  std::lock_guard<std::mutex> lock(g_scan_ws_mutex);
  ScanWsEntry& ent = g_scan_ws[dev];
  if (!have_ctx || ent.addr == nullptr || ent.ctx != ctx) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_nbgrid_scan_ws);
    if (e != cudaSuccess || p == nullptr) {
      char msg[256];
      snprintf(msg, sizeof(msg), "att_nbgrid_count_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
               cudaGetErrorString(e));
      return att::report_error(ATT_E_CUDA, msg);
    }
    ent.addr = p;
    ent.ctx = have_ctx ? ctx : nullptr;
  }
  *out = ent.addr;
  return ATT_OK;
}
}  // namespace

extern "C" int att_nbgrid_count_noalloc(const AttGridGeom* geom, const float* rec_dev, int n_rec, float radius,
                                        uint32_t* hdr_dev, unsigned long long* total_dev, void* stream) {
  char msg[256];
  int rc = att::check_geom(geom);  // the same geometry rules as att_nbgrid_count
  if (rc != ATT_OK) return rc;
  const long long nvox = (long long)geom->dim[0] * geom->dim[1] * geom->dim[2];
  if (nvox > ATT_NBGRID_NOALLOC_MAX_VOXELS) {
    snprintf(msg, sizeof(msg),
             "att_nbgrid_count_noalloc: %lld grid points exceed the fixed workspace (at most %lld); "
             "use att_nbgrid_count with a caller-provided workspace",
             nvox, (long long)ATT_NBGRID_NOALLOC_MAX_VOXELS);
    return att::report_error(ATT_E_INVALID, msg);
  }
  if (n_rec < 0 || n_rec >= (int)ATT_NB_EMPTY || (n_rec > 0 && rec_dev == nullptr))
    return att::report_error(ATT_E_INVALID, "att_nbgrid_count_noalloc: receptor beads");
  if (hdr_dev == nullptr || total_dev == nullptr)
    return att::report_error(ATT_E_INVALID, "att_nbgrid_count_noalloc: NULL output");
  if (!(radius >= 0.f)) return att::report_error(ATT_E_INVALID, "att_nbgrid_count_noalloc: radius < 0");
  void* ws = nullptr;
  rc = scan_ws_address(&ws);
  if (rc != ATT_OK) return rc;
  // every workspace word the scan reads is written by the count kernel of the
  // same call first, so nothing has to be cleared between calls
  cudaError_t e = att::launch_nb_count(*geom, rec_dev, n_rec, radius, hdr_dev, total_dev, ws, (cudaStream_t)stream);
  if (e != cudaSuccess) {
    snprintf(msg, sizeof(msg), "att_nbgrid_count_noalloc: %s", cudaGetErrorString(e));
    return att::report_error(ATT_E_CUDA, msg);
  }
  return ATT_OK;
}
