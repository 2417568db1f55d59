// fsl_noalloc.cu -- a cell-list build that allocates no device memory.
//
// fsl_cell_list needs a handle, and fsl_create allocates the handle's device
// buffers with cudaMalloc.  Some callers cannot do that:
//   * a host framework that owns all device memory through its own pool and
//     only hands out buffers it allocated itself;
//   * a loop that keeps other work in flight on the GPU and must not stall
//     it: cudaMalloc and cudaFree can synchronise the whole device.
// fsl_cell_list_noalloc serves them: the caller passes the positions and the
// three output arrays in device memory it already owns, and the counting
// sort's scratch (per-cell counters, the unordered bucket array, the scan's
// block totals) lives in the file-scope arrays below.  Those arrays are part
// of the library image: every GPU that loads the library holds them (about
// 9 MiB) until the process exits, whether or not this entry point is called.
#include <cstdio>
#include <mutex>

#include "../../include/fluamsl.h"
#include "fsl_internal.cuh"

namespace {

constexpr int kMaxCells = 1 << 20;      // neighbour-grid cells (m^3)
constexpr int kMaxParticles = 1 << 18;  // particles
constexpr int kScanTile = 4096;         // elements per block of the scan
constexpr int kMaxScanBlocks = (kMaxCells + kScanTile - 1) / kScanTile;

static __device__ __align__(256) int g_cnt[kMaxCells];
static __device__ __align__(256) int g_fill[kMaxCells];
static __device__ __align__(256) int g_tmp[kMaxParticles];
static __device__ __align__(256) int g_bsum[kMaxScanBlocks + 1];
static __device__ __align__(256) int g_err[4];

// Device addresses of the arrays, looked up once per device.  In host code
// the names above are host-side stand-ins, not device addresses.
struct Scratch {
  int *cnt = nullptr, *fill = nullptr, *tmp = nullptr, *bsum = nullptr, *err = nullptr;
  bool ready = false;
};
constexpr int kMaxDevices = 64;
Scratch g_scratch[kMaxDevices];
std::mutex g_mutex;

int fail(int code, const char* msg) { return fsl::set_last_error(code, msg); }

int scratch_for_current_device(Scratch** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(FSL_E_CUDA, "fsl_cell_list_noalloc: no current CUDA device");
  std::lock_guard<std::mutex> lock(g_mutex);
  Scratch& s = g_scratch[dev];
  if (!s.ready) {
    if (cudaGetSymbolAddress((void**)&s.cnt, g_cnt) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&s.fill, g_fill) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&s.tmp, g_tmp) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&s.bsum, g_bsum) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&s.err, g_err) != cudaSuccess) {
      cudaGetLastError();
      return fail(FSL_E_CUDA, "fsl_cell_list_noalloc: cudaGetSymbolAddress failed");
    }
    s.ready = true;
  }
  *out = &s;
  return FSL_OK;
}

}  // namespace

extern "C" int fsl_cell_list_noalloc(double lx, double ly, double lz, double cutoff, int64_t np,
                                     const double* q_dev, int32_t* cell_of_dev,
                                     int32_t* start_dev, int32_t* sorted_dev, void* stream) {
  if (!(lx > 0 && ly > 0 && lz > 0)) return fail(FSL_E_ARG, "box lengths must be > 0");
  if (!(cutoff > 0)) return fail(FSL_E_ARG, "cutoff must be > 0");
  if (np < 0 || np > kMaxParticles)
    return fail(FSL_E_ARG, "fsl_cell_list_noalloc: at most 262144 particles");
  if (np > 0 && (!q_dev || !cell_of_dev || !sorted_dev)) return fail(FSL_E_ARG, "null array");
  if (!start_dev) return fail(FSL_E_ARG, "null start array");
  // neighbour grid of the reference, src/createBoundariesRK2GPU.cu:134-141
  double mxd = lx / cutoff, myd = ly / cutoff, mzd = lz / cutoff;
  if (mxd > 1e6 || myd > 1e6 || mzd > 1e6)
    return fail(FSL_E_ARG, "fsl_cell_list_noalloc: at most 1048576 neighbour-grid cells");
  fsl::Params P{};
  P.mnx = (int)mxd < 3 ? 3 : (int)mxd;
  P.mny = (int)myd < 3 ? 3 : (int)myd;
  P.mnz = (int)mzd < 3 ? 3 : (int)mzd;
  if ((int64_t)P.mnx * P.mny * P.mnz > kMaxCells)
    return fail(FSL_E_ARG, "fsl_cell_list_noalloc: at most 1048576 neighbour-grid cells");
  P.mN = P.mnx * P.mny * P.mnz;
  P.lx = lx;
  P.ly = ly;
  P.lz = lz;
  P.invlx = 1. / lx;
  P.invly = 1. / ly;
  P.invlz = 1. / lz;
  P.invdnx = double(P.mnx) / lx;
  P.invdny = double(P.mny) / ly;
  P.invdnz = double(P.mnz) / lz;
  P.np = (int)np;
  Scratch* s = nullptr;
  int rc = scratch_for_current_device(&s);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // the counters start at zero; the unordered buckets and block totals are
  // fully rewritten before they are read.  A single instance travels to the
  // kernels as a by-value argument: nothing to allocate or copy first.
  fsl::Rep r{};
  r.P = P;
  r.active = 1;
  r.q = const_cast<double*>(q_dev);
  r.cell_of = cell_of_dev;
  r.start = start_dev;
  r.sorted = sorted_dev;
  r.cnt = s->cnt;
  r.fill = s->fill;
  r.tmp = s->tmp;
  r.bsum = s->bsum;
  r.err = s->err;
  fsl::Batch B{};
  B.one = &r;
  B.nrep = 1;
  B.mN = P.mN;
  B.max_np = P.np;
  fsl::launch_cells(B, 0, st);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(FSL_E_CUDA, cudaGetErrorString(e));
  return FSL_OK;
}
