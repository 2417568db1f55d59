// cuda_host_shim.h -- lets the reference's own Stokes-limit CUDA sources
// (fbusabiaga/fluam src/*.cu) compile and run on the host, serially, as a
// pinning reference for the FP64 oracle.  TEST INFRASTRUCTURE ONLY.
//
// What it stands in for:
//   * CUDA qualifiers and launches: kernels become plain functions; a launch
//     runs every (block, thread) in order, one at a time, so the atomics of
//     the reference append to its lists in ascending thread order;
//   * the runtime: device memory is host memory (malloc), copies are memcpy,
//     __constant__ symbols are ordinary globals;
//   * legacy texture references: a bound pointer; tex1Dfetch is an index,
//     fetch_double reads the bound double array, and tex1D on the normalised,
//     clamped, linear-filtered LJ force table uses the texture unit's rule
//     (x_B = x N - 1/2, fractional weight with 8 fractional bits, rounded to
//     nearest), the same rule the oracle and the CUDA path use;
//   * cuFFT: cufftExecZ2Z is a direct O(m^2)-per-line separable DFT with the
//     cuFFT sign convention (forward -1, inverse +1, unnormalised);
//   * cuRAND: curandGenerateNormalDouble fills the array with the counter-based
//     Philox normals of the oracle (orc_noise), draw number = call number.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__
#define __forceinline__ inline

struct int2 { int x, y; };
struct float2 { float x, y; };
struct double2 { double x, y; };
struct dim3 {
  unsigned x = 1, y = 1, z = 1;
  dim3() {}
  dim3(unsigned a, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
extern dim3 blockIdx, blockDim, threadIdx, gridDim;

typedef int cudaError_t;
enum { cudaSuccess = 0 };
enum cudaMemcpyKind { cudaMemcpyHostToHost, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost,
                      cudaMemcpyDeviceToDevice };
enum cudaTextureFilterMode { cudaFilterModePoint = 0, cudaFilterModeLinear = 1 };
enum cudaTextureAddressMode { cudaAddressModeWrap = 0, cudaAddressModeClamp = 1,
                              cudaAddressModeMirror = 2, cudaAddressModeBorder = 3 };
enum cudaTextureReadMode { cudaReadModeElementType = 0 };
enum cudaChannelFormatKind { cudaChannelFormatKindSigned, cudaChannelFormatKindUnsigned,
                             cudaChannelFormatKindFloat };
struct cudaChannelFormatDesc { int x, y, z, w; cudaChannelFormatKind f; };
inline cudaChannelFormatDesc cudaCreateChannelDesc(int x, int y, int z, int w,
                                                   cudaChannelFormatKind f) {
  return {x, y, z, w, f};
}
struct cudaArray { std::vector<float> data; };

inline const char* cudaGetErrorString(cudaError_t) { return "no error"; }
inline cudaError_t cudaMalloc(void** p, size_t n) {
  *p = calloc(n ? n : 1, 1);
  return *p ? cudaSuccess : 2;
}
inline cudaError_t cudaFree(void* p) {
  free(p);
  return cudaSuccess;
}
inline cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) {
  memmove(d, s, n);
  return cudaSuccess;
}
inline cudaError_t cudaMemset(void* d, int v, size_t n) {
  memset(d, v, n);
  return cudaSuccess;
}
template <class T>
cudaError_t cudaMemcpyToSymbol(T& sym, const void* src, size_t n, size_t off = 0,
                               cudaMemcpyKind = cudaMemcpyHostToDevice) {
  memcpy(reinterpret_cast<char*>(&sym) + off, src, n);
  return cudaSuccess;
}
template <class T>
cudaError_t cudaMemcpyFromSymbol(void* dst, const T& sym, size_t n, size_t off = 0,
                                 cudaMemcpyKind = cudaMemcpyDeviceToHost) {
  memcpy(dst, reinterpret_cast<const char*>(&sym) + off, n);
  return cudaSuccess;
}
inline cudaError_t cudaMallocArray(cudaArray** a, const cudaChannelFormatDesc*, size_t w,
                                   size_t = 1) {
  *a = new cudaArray();
  (*a)->data.assign(w, 0.0f);
  return cudaSuccess;
}
inline cudaError_t cudaMemcpyToArray(cudaArray* a, size_t, size_t, const void* src, size_t n,
                                     cudaMemcpyKind) {
  memcpy(a->data.data(), src, n);
  return cudaSuccess;
}
inline cudaError_t cudaFreeArray(cudaArray* a) {
  delete a;
  return cudaSuccess;
}
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
inline cudaError_t cudaThreadSynchronize() { return cudaSuccess; }
inline cudaError_t cudaSetDevice(int) { return cudaSuccess; }
inline cudaError_t cudaGetDevice(int* d) {
  *d = 0;
  return cudaSuccess;
}
inline cudaError_t cudaGetDeviceCount(int* n) {
  *n = 1;
  return cudaSuccess;
}
inline cudaError_t cudaDriverGetVersion(int* v) {
  *v = 0;
  return cudaSuccess;
}
inline cudaError_t cudaRuntimeGetVersion(int* v) {
  *v = 0;
  return cudaSuccess;
}
struct cudaDeviceProp {
  char name[256] = "host emulation of the reference kernels";
  int major = 0, minor = 0, multiProcessorCount = 1, regsPerBlock = 0, warpSize = 1,
      maxThreadsPerBlock = 1, clockRate = 0, computeMode = 0;
  size_t totalGlobalMem = 0, totalConstMem = 0, sharedMemPerBlock = 0;
};
inline cudaError_t cudaGetDeviceProperties(cudaDeviceProp* p, int) {
  *p = cudaDeviceProp();
  return cudaSuccess;
}
inline cudaError_t cudaGetLastError() { return cudaSuccess; }

// ------------------------------------------------------------- textures ---
template <class T, int dim = 1, int mode = cudaReadModeElementType>
struct texture {
  int normalized = 0;
  int filterMode = 0;
  int addressMode[3] = {0, 0, 0};
  const T* ptr = nullptr;
  size_t n = 0;
};
void shim_bad_fetch(const char* what, long i, long n);
template <class T, int d, int m>
inline T tex1Dfetch(const texture<T, d, m>& t, int i) {
  if (i < 0 || (size_t)i >= t.n) shim_bad_fetch("tex1Dfetch", i, (long)t.n);
  return t.ptr[i];
}
template <class T, int d, int m, class P>
cudaError_t cudaBindTexture(size_t*, texture<T, d, m>& t, const P* ptr, size_t bytes) {
  t.ptr = reinterpret_cast<const T*>(ptr);
  t.n = bytes / sizeof(T);
  return cudaSuccess;
}
template <class T, int d, int m>
cudaError_t cudaUnbindTexture(texture<T, d, m>& t) {
  t.ptr = nullptr;
  t.n = 0;
  return cudaSuccess;
}
template <class T, int d, int m>
cudaError_t cudaBindTextureToArray(texture<T, d, m>& t, cudaArray* a, cudaChannelFormatDesc) {
  t.ptr = reinterpret_cast<const T*>(a->data.data());
  t.n = a->data.size();
  return cudaSuccess;
}
// normalised coordinates, clamp, point or linear filtering
template <int d, int m>
inline float tex1D(const texture<float, d, m>& t, float x) {
  const int N = (int)t.n;
  const float* T = t.ptr;
  if (t.filterMode == cudaFilterModePoint) {
    double xb = t.normalized ? (double)x * N : (double)x;
    int i = (int)std::floor(xb);
    i = i < 0 ? 0 : (i > N - 1 ? N - 1 : i);
    return T[i];
  }
  double xb = (t.normalized ? (double)x * N : (double)x) - 0.5;
  double fl = std::floor(xb);
  int i = (int)fl;
  float a = (float)(std::nearbyint((xb - fl) * 256.0) / 256.0);
  int i0 = i < 0 ? 0 : (i > N - 1 ? N - 1 : i);
  int i1 = i + 1 < 0 ? 0 : (i + 1 > N - 1 ? N - 1 : i + 1);
  return (1.0f - a) * T[i0] + a * T[i1];
}
inline double fetch_double(const texture<int2, 1>& t, int i) {
  // an int2 texel holds one double
  if (i < 0 || (size_t)i >= t.n) shim_bad_fetch("fetch_double", i, (long)t.n);
  return reinterpret_cast<const double*>(t.ptr)[i];
}

// ------------------------------------------------------------ math -------
// CUDA's double reciprocal square root, as 1 / sqrt on the host (the
// quasi-2D kernels use it; within an ulp or two of the device function)
inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }

// -------------------------------------------------------------- atomics ---
inline int atomicAdd(int* p, int v) {
  int o = *p;
  *p += v;
  return o;
}
inline double atomicAdd(double* p, double v) {
  double o = *p;
  *p += v;
  return o;
}

// ------------------------------------------------------------- launches ---
// SHIM_LAUNCH(grid, block, call): every block and thread of the launch, in
// order, with blockIdx / threadIdx set.
#define SHIM_LAUNCH(G, B, CALL)                                              \
  do {                                                                       \
    dim3 shim_g_(G), shim_b_(B);                                             \
    gridDim = shim_g_;                                                       \
    blockDim = shim_b_;                                                      \
    for (unsigned shim_bx = 0; shim_bx < shim_g_.x; ++shim_bx)               \
      for (unsigned shim_tx = 0; shim_tx < shim_b_.x; ++shim_tx) {           \
        blockIdx = dim3(shim_bx);                                            \
        threadIdx = dim3(shim_tx);                                           \
        CALL;                                                                \
      }                                                                      \
  } while (0)

// ---------------------------------------------------------------- cuFFT ---
typedef int cufftHandle;
typedef int cufftResult;
typedef double2 cufftDoubleComplex;
typedef float2 cufftComplex;
typedef double cufftDoubleReal;
enum { CUFFT_SUCCESS = 0 };
enum cufftType { CUFFT_R2C = 0x2a, CUFFT_C2R = 0x2c, CUFFT_C2C = 0x29, CUFFT_D2Z = 0x6a,
                 CUFFT_Z2D = 0x6c, CUFFT_Z2Z = 0x69 };
#define CUFFT_FORWARD -1
#define CUFFT_INVERSE 1
cufftResult cufftPlan3d(cufftHandle* plan, int nx, int ny, int nz, cufftType type);
cufftResult cufftPlan2d(cufftHandle* plan, int nx, int ny, cufftType type);
cufftResult cufftExecZ2Z(cufftHandle plan, cufftDoubleComplex* in, cufftDoubleComplex* out,
                         int direction);
cufftResult cufftDestroy(cufftHandle plan);

// --------------------------------------------------------------- cuRAND ---
typedef int curandGenerator_t;
typedef int curandStatus_t;
enum curandRngType { CURAND_RNG_PSEUDO_DEFAULT = 100 };
curandStatus_t curandCreateGenerator(curandGenerator_t* g, curandRngType);
curandStatus_t curandSetPseudoRandomGeneratorSeed(curandGenerator_t g, unsigned long long seed);
curandStatus_t curandGenerateNormalDouble(curandGenerator_t g, double* out, size_t n, double mean,
                                          double stddev);
curandStatus_t curandDestroyGenerator(curandGenerator_t g);

// cutilSafeCall of src/GPU.cu:28-35
#define cutilSafeCall(i) (void)(i)
