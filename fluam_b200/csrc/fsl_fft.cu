// fsl_fft.cu -- the periodic Stokes solve of the Stokes-limit step:
//   W = f + c div(Sigma)  ->  forward FFT  ->  shift, projection, 1/(eta k^2),
//   unshift  ->  inverse FFT  ->  v
// (src/runSchemeStokesLimit.cu:186-214 and 234-261; kernels
// kernelConstructWstokesLimit(_2), kernelShift, kernelUpdateVstokesLimit,
// doubleComplexToDoubleNormalized).  The reference runs 3 + 3 cuFFT Z2Z
// transforms and 5 elementwise passes per solve in FP64; here the transform is
// a hand-written FP32 mixed-radix Stockham FFT in shared memory, done as
// passes over the half spectrum:
//   k_wbuild    builds W from the fixed-point spread field and the noise;
//   k_plane_fwd 2-D real-to-complex transform of one xy plane per block;
//   k_zsolve    transforms along z, applies the spectral multiplier to all
//               three components of each mode, and transforms back along z;
//   k_plane_inv 2-D complex-to-real transform of one xy plane per block.
// Planes too large for shared memory take five passes instead (k_xfwd,
// k_yfft, k_zsolve, k_yfft, k_xinv).  Every kernel serves a batch of
// instances of one size class; the grid's last dimension picks the instance.
// The multiplier keeps Hermitian symmetry (the sign of sin(pi j/m) for
// j > m/2 cancels between gradient and shift), so the real-to-complex form
// equals the reference's Re(IFFT(...)) up to rounding.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <vector>

#include <algorithm>
#include "fsl_internal.cuh"

namespace fsl {

struct Radices {
  int n;
  int nst;
  int r[14];
};

constexpr int kMaxZCand = 6;
constexpr int kMaxPCand = 4;

struct FftPlan {
  Radices rx, ry, rz;
  float2 *twx = nullptr, *twy = nullptr, *twz = nullptr;  // exp(-2 pi i t / m)
  // sin(pi j / m); the kernel multiplies by the instance's 2/h, so one table
  // serves every instance of a size class whatever its box
  float *sx = nullptr, *sy = nullptr, *sz = nullptr;
  float2 *ex = nullptr, *ey = nullptr, *ez = nullptr;  // exp(+i pi j / m)
  size_t smem_x = 0, smem_y = 0, smem_z = 0, smem_plane = 0;
  bool use_plane = false;  // whole-plane kernels fit in shared memory
  bool ok = false;
  // kernel instances: compiled sizes when available, else runtime sizes;
  // [0] batched, [1] single instance
  void (*plane_fwd[2])(RepSrc, Rep, Radices, Radices, const float2*, const float2*) = {};
  void (*plane_inv[2])(RepSrc, Rep, Radices, Radices, const float2*, const float2*) = {};
  void (*zsolve[2])(RepSrc, Rep, Radices, const float2*, const float*, const float*, const float*,
                    const float2*, const float2*, const float2*) = {};
  // register-resident passes for compiled edges (null: not available)
  void (*plane_fwd_r[2])(RepSrc, Rep, const float2*) = {};
  void (*plane_inv_r[2])(RepSrc, Rep, const float2*) = {};
  void (*zsolve_r[2])(RepSrc, Rep, const float2*, const float*, const float*, const float*,
                      const float2*, const float2*, const float2*) = {};
  // the same transform as five passes of warp tasks (fsl_fft_lines.cuh);
  // null where the edge's lines do not fit in a warp
  void (*line_xf[2])(RepSrc, Rep, const float2*) = {};
  void (*line_yf[2])(RepSrc, Rep, const float2*) = {};
  void (*line_yi[2])(RepSrc, Rep, const float2*) = {};
  void (*line_xi[2])(RepSrc, Rep, const float2*) = {};
  int line_lw = 0;          // lines per warp
  size_t smem_lines = 0;
  bool use_lines = false;   // the five-pass schedule (picked by fft_autotune)
  float sched_us[2] = {};   // measured solve transform time: plane, lines
  int plane_pb = 0, plane_threads = 0;      // planes per block, threads per block
  int z_kx = 0, z_ky = 0, z_threads = 0;    // zsolve tile and threads per block
  size_t smem_plane_r = 0, smem_z_r = 0;
  // tile candidates of the register z pass (same arithmetic, other (kx, ky)
  // tiles per block); the first is the default, fft_autotune picks one
  struct ZCand {
    void (*k[2])(RepSrc, Rep, const float2*, const float*, const float*, const float*, const float2*,
                 const float2*, const float2*);
    int kx, ky, threads;
    size_t smem;
  } zc[kMaxZCand];
  int nzc = 0;
  bool tuned = false;
  float zc_us[kMaxZCand] = {};  // measured time per candidate (us per launch)
  // planes-per-block candidates of the register plane passes (same
  // arithmetic, another number of independent planes per block); the first
  // is the default, fft_autotune picks one
  struct PCand {
    void (*fwd[2])(RepSrc, Rep, const float2*);
    void (*inv[2])(RepSrc, Rep, const float2*);
    int pb, threads;
    size_t smem;
  } pc[kMaxPCand];
  int npc = 0;
  float pc_us[kMaxPCand] = {};  // measured plane-schedule transform per candidate (us)
};

static bool factorize(int n, Radices& R) {
  R.n = n;
  R.nst = 0;
  int m = n;
  while (m % 4 == 0 && R.nst < 14) {
    R.r[R.nst++] = 4;
    m /= 4;
  }
  const int ps[5] = {2, 3, 5, 7, 11};
  for (int pi = 0; pi < 5; ++pi)
    while (m % ps[pi] == 0 && R.nst < 14) {
      R.r[R.nst++] = ps[pi];
      m /= ps[pi];
    }
  return m == 1;
}

// p-point DFT coefficients exp(-2 pi i t / p) for p = 5, 7, 11
__constant__ float2 c_w5[5];
__constant__ float2 c_w7[7];
__constant__ float2 c_w11[11];

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// V[q] = sum_r v[r] exp(dir 2 pi i r q / P)
template <int P>
__device__ __forceinline__ void dft(float2 (&v)[P], int dir);

template <>
__device__ __forceinline__ void dft<2>(float2 (&v)[2], int) {
  float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <>
__device__ __forceinline__ void dft<4>(float2 (&v)[4], int dir) {
  float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
  float2 c = cadd(v[1], v[3]), e = csub(v[1], v[3]);
  float2 d = make_float2(-dir * e.y, dir * e.x);  // (dir i) e
  v[0] = cadd(a, c);
  v[2] = csub(a, c);
  v[1] = cadd(b, d);
  v[3] = csub(b, d);
}

template <>
__device__ __forceinline__ void dft<3>(float2 (&v)[3], int dir) {
  const float s = 0.86602540378443864676f * dir;  // dir sqrt(3)/2
  float2 t1 = cadd(v[1], v[2]);
  float2 t2 = csub(v[1], v[2]);
  float2 m = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
  float2 r = make_float2(-s * t2.y, s * t2.x);  // (i s) t2
  v[0] = cadd(v[0], t1);
  v[1] = cadd(m, r);
  v[2] = csub(m, r);
}

template <int P>
__device__ __forceinline__ void dft_generic(float2 (&v)[P], int dir, const float2* w) {
  float2 out[P];
#pragma unroll
  for (int q = 0; q < P; ++q) {
    float2 acc = v[0];
#pragma unroll
    for (int r = 1; r < P; ++r) {
      float2 t = w[(r * q) % P];
      if (dir > 0) t.y = -t.y;
      acc = cadd(acc, cmul(v[r], t));
    }
    out[q] = acc;
  }
#pragma unroll
  for (int q = 0; q < P; ++q) v[q] = out[q];
}

template <>
__device__ __forceinline__ void dft<5>(float2 (&v)[5], int dir) { dft_generic<5>(v, dir, c_w5); }
template <>
__device__ __forceinline__ void dft<7>(float2 (&v)[7], int dir) { dft_generic<7>(v, dir, c_w7); }
template <>
__device__ __forceinline__ void dft<11>(float2 (&v)[11], int dir) { dft_generic<11>(v, dir, c_w11); }

// One Stockham stage of radix P on nlines lines of length n stored in shared
// memory with element k of line l at [k * LS + l]; Ns is the length of the
// sub-transforms already done.  tw[t] = exp(-2 pi i t / n).
template <int P>
__device__ __forceinline__ void stage(const float2* __restrict__ A, float2* __restrict__ B, int n,
                                      int LS, int nlines, int Ns, const float2* __restrict__ tw,
                                      int dir) {
  const int nbut = n / P;
  const int tstride = n / (Ns * P);
  const int total = nbut * nlines;
  for (int w = threadIdx.x; w < total; w += blockDim.x) {
    int l = w % nlines, j = w / nlines;
    int k = j % Ns;
    float2 v[P];
#pragma unroll
    for (int r = 0; r < P; ++r) v[r] = A[(j + r * nbut) * LS + l];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < P; ++r) {
        float2 t = tw[r * k * tstride];
        if (dir > 0) t.y = -t.y;
        v[r] = cmul(v[r], t);
      }
    }
    dft<P>(v, dir);
    int base = (j - k) * P + k;
#pragma unroll
    for (int r = 0; r < P; ++r) B[(base + r * Ns) * LS + l] = v[r];
  }
}

// Full transform; returns the buffer (A or B) that holds the result.
__device__ float2* fft_lines(float2* A, float2* B, int LS, int nlines, const Radices& R,
                             const float2* tw, int dir) {
  int Ns = 1;
  for (int s = 0; s < R.nst; ++s) {
    int p = R.r[s];
    switch (p) {
      case 4: stage<4>(A, B, R.n, LS, nlines, Ns, tw, dir); break;
      case 2: stage<2>(A, B, R.n, LS, nlines, Ns, tw, dir); break;
      case 3: stage<3>(A, B, R.n, LS, nlines, Ns, tw, dir); break;
      case 5: stage<5>(A, B, R.n, LS, nlines, Ns, tw, dir); break;
      case 7: stage<7>(A, B, R.n, LS, nlines, Ns, tw, dir); break;
      default: stage<11>(A, B, R.n, LS, nlines, Ns, tw, dir); break;
    }
    __syncthreads();
    float2* t = A;
    A = B;
    B = t;
    Ns *= p;
  }
  return A;
}

// Compile-time variant of `stage` / `fft_lines`: with the size, radix
// schedule, line count and stride known to the compiler, the index
// arithmetic folds into shifts and multiplies.
template <int N, int P, int NS, int NL, int LS>
__device__ __forceinline__ void stage_ct(const float2* __restrict__ A, float2* __restrict__ B,
                                         const float2* __restrict__ tw, int dir) {
  constexpr int NBUT = N / P;
  constexpr int TOT = NBUT * NL;
  constexpr int TSTRIDE = N / (NS * P);
  for (int w = threadIdx.x; w < TOT; w += blockDim.x) {
    const int l = w % NL, j = w / NL;
    const int k = j % NS;
    float2 v[P];
#pragma unroll
    for (int r = 0; r < P; ++r) v[r] = A[(j + r * NBUT) * LS + l];
    if (NS > 1) {
#pragma unroll
      for (int r = 1; r < P; ++r) {
        float2 t = tw[r * k * TSTRIDE];
        if (dir > 0) t.y = -t.y;
        v[r] = cmul(v[r], t);
      }
    }
    dft<P>(v, dir);
    const int base = (j - k) * P + k;
#pragma unroll
    for (int r = 0; r < P; ++r) B[(base + r * NS) * LS + l] = v[r];
  }
}

template <int N, int NL, int LS, int NS, int... Rs>
struct FftCT;
template <int N, int NL, int LS, int NS>
struct FftCT<N, NL, LS, NS> {
  __device__ static float2* run(float2* A, float2*, const float2*, int) { return A; }
};
template <int N, int NL, int LS, int NS, int P0, int... Rs>
struct FftCT<N, NL, LS, NS, P0, Rs...> {
  __device__ static float2* run(float2* A, float2* B, const float2* tw, int dir) {
    stage_ct<N, P0, NS, NL, LS>(A, B, tw, dir);
    __syncthreads();
    return FftCT<N, NL, LS, NS * P0, Rs...>::run(B, A, tw, dir);
  }
};

// sizes with a compiled radix schedule; others use the runtime transform
__host__ __device__ constexpr bool fft_ct_size(int n) {
  return n == 16 || n == 24 || n == 32 || n == 48 || n == 64 || n == 96 || n == 128 || n == 256;
}

template <int N, int NL, int LS>
__device__ __forceinline__ float2* fft_ct(float2* A, float2* B, const float2* tw, int dir) {
  if constexpr (N == 256) return FftCT<N, NL, LS, 1, 4, 4, 4, 4>::run(A, B, tw, dir);
  else if constexpr (N == 128) return FftCT<N, NL, LS, 1, 4, 4, 4, 2>::run(A, B, tw, dir);
  else if constexpr (N == 96) return FftCT<N, NL, LS, 1, 4, 4, 3, 2>::run(A, B, tw, dir);
  else if constexpr (N == 64) return FftCT<N, NL, LS, 1, 4, 4, 4>::run(A, B, tw, dir);
  else if constexpr (N == 48) return FftCT<N, NL, LS, 1, 4, 4, 3>::run(A, B, tw, dir);
  else if constexpr (N == 32) return FftCT<N, NL, LS, 1, 4, 4, 2>::run(A, B, tw, dir);
  else if constexpr (N == 24) return FftCT<N, NL, LS, 1, 4, 3, 2>::run(A, B, tw, dir);
  else return FftCT<N, NL, LS, 1, 4, 4>::run(A, B, tw, dir);  // 16
}

// N > 0: compiled schedule; N == 0: runtime radices R (any 2,3,5,7,11-smooth n)
template <int N, int NL, int LS>
__device__ __forceinline__ float2* fft_any(float2* A, float2* B, const Radices& R,
                                           const float2* tw, int dir) {
  if constexpr (N > 0) return fft_ct<N, NL, LS>(A, B, tw, dir);
  else return fft_lines(A, B, LS, NL, R, tw, dir);
}

constexpr int kXPairs = 16;  // x pass: row pairs (complex lines) per block
constexpr int kYTile = 16;   // y pass: kx columns per block
constexpr int kZTile = 8;    // z pass: kx columns per block (x 3 components)
constexpr int kFftThreads = 512;

// W = f + c div(Sigma) of all three components of every cell
// (src/stokesLimitFunctions.cu:2281-2378, 3922-4069): the fixed-point spread
// field times 2^-40/dV plus c times the stochastic stress divergence that
// k_div wrote (D1 = div Sigma_1 for one stress sample, D12 =
// div(Sigma_1 + Sigma_2) for two), with c = sqrt(2) (midpoint, one sample),
// sqrt(1/2) (two samples) or 1 (first-order scheme,
// src/runSchemeStokesLimitFirstOrder.cu:181-190).  The spread field is
// cleared behind the read, ready for the next spread.  One thread per cell:
// the loads of a warp are coalesced rows, full occupancy.
template <bool ONE>
__global__ void k_wbuild(FSL_KARGS, int nsets, double nfac, int clear) {
  FSL_REP_AT(blockIdx.y);
  const float scale = (float)(kFixedInv / P.dV);
  const float fac = (float)nfac;
  const size_t nc = (size_t)P.nc;
  const float* D = R.ndiv + (nsets > 1 ? 3 * nc : 0);
  // float-atomic form: FP32 sums in the first 3 nc floats of the buffer
  const bool fatom = P.prec == PREC_FLOAT;
  float* gf = reinterpret_cast<float*>(R.grid);
  const float fscale = (float)(1.0 / P.dV);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nc;
       i += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      float w;
      const float d = __ldg(D + comp * nc + i);
      if (fatom) {
        w = w_float(gf[comp * nc + i], fscale, fac, d);
        if (clear) gf[comp * nc + i] = 0.0f;
      } else {
        w = w_fixed((long long)R.grid[comp * nc + i], scale, fac, d);
        if (clear) R.grid[comp * nc + i] = 0ull;
      }
      R.wbuf[comp * nc + i] = w;
    }
  }
}

// Zeroes the spread field (3 nc 64-bit sums, or 3 nc floats of the
// float-atomic form) with streaming stores, which leave the L2 to the
// transforms it runs beside.
template <bool ONE>
__global__ void k_field_clear(FSL_KARGS) {
  FSL_REP_AT(blockIdx.y);
  const size_t bytes = (size_t)3 * P.nc * (P.prec == PREC_FLOAT ? 4 : 8);
  float4* q = reinterpret_cast<float4*>(R.grid);
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < bytes / 16; i += (size_t)gridDim.x * blockDim.x)
    __stcs(q + i, z);
}

// k_wbuild for mx a multiple of 4: one thread per four x cells, 16-byte loads
// of the fixed-point field, the noise rows and W, and 16-byte clears.
template <bool ONE>
__global__ void k_wbuild4(FSL_KARGS, int nsets, double nfac, int clear) {
  FSL_REP_AT(blockIdx.y);
  const float scale = (float)(kFixedInv / P.dV);
  const float fac = (float)nfac;
  const size_t nc = (size_t)P.nc;
  const float* D = R.ndiv + (nsets > 1 ? 3 * nc : 0);
  const size_t ng = nc >> 2;
  const bool fatom = P.prec == PREC_FLOAT;
  float* gf = reinterpret_cast<float*>(R.grid);
  const float fscale = (float)(1.0 / P.dV);
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < ng;
       g += (size_t)gridDim.x * blockDim.x) {
    const size_t i0 = g << 2;
    float w[3][4];
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      const float4 d = __ldg(reinterpret_cast<const float4*>(D + comp * nc + i0));
      if (fatom) {
        float4* fp = reinterpret_cast<float4*>(gf + comp * nc + i0);
        const float4 ga = *fp;
        w[comp][0] = w_float(ga.x, fscale, fac, d.x);
        w[comp][1] = w_float(ga.y, fscale, fac, d.y);
        w[comp][2] = w_float(ga.z, fscale, fac, d.z);
        w[comp][3] = w_float(ga.w, fscale, fac, d.w);
        if (clear) *fp = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        continue;
      }
      const longlong2* gp = reinterpret_cast<const longlong2*>(R.grid + comp * nc + i0);
      const longlong2 ga = gp[0], gb = gp[1];
      w[comp][0] = w_fixed(ga.x, scale, fac, d.x);
      w[comp][1] = w_fixed(ga.y, scale, fac, d.y);
      w[comp][2] = w_fixed(gb.x, scale, fac, d.z);
      w[comp][3] = w_fixed(gb.y, scale, fac, d.w);
    }
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      *reinterpret_cast<float4*>(R.wbuf + comp * nc + i0) =
          make_float4(w[comp][0], w[comp][1], w[comp][2], w[comp][3]);
      if (fatom || !clear) continue;  // cleared at the read, or by k_field_clear
      longlong2* gq = reinterpret_cast<longlong2*>(R.grid + comp * nc + i0);
      gq[0] = make_longlong2(0, 0);
      gq[1] = make_longlong2(0, 0);
    }
  }
}

// Real-to-complex transform along x of W.  Block (bx, comp, instance)
// handles the row pairs [bx*kXPairs, ...); row R = y + my z; the pair
// (2p, 2p+1) is transformed as the complex line row_2p + i row_2p+1.
template <bool ONE>
__global__ void __launch_bounds__(kFftThreads)
    k_xfwd(FSL_KARGS, Radices Rx, const float2* __restrict__ tw) {
  FSL_REP_AT(blockIdx.z);
  extern __shared__ float2 smem[];
  const int mx = P.mx, mxh = P.mxh;
  const int LS = kXPairs + 1;
  float2* A = smem;
  float2* B = A + mx * LS;
  float2* stw = B + mx * LS;
  const int comp = blockIdx.y;
  const int nrows = P.my * P.mz;
  const int row0 = blockIdx.x * 2 * kXPairs;
  for (int t = threadIdx.x; t < mx; t += blockDim.x) stw[t] = tw[t];
  const float* W = R.wbuf + (size_t)comp * P.nc;
  float* Af = reinterpret_cast<float*>(A);
  for (int e = threadIdx.x; e < 2 * kXPairs * mx; e += blockDim.x) {
    int rl = e / mx, x = e - rl * mx;
    int Rw = row0 + rl;
    float w = Rw < nrows ? W[x + (size_t)mx * Rw] : 0.0f;
    Af[2 * (x * LS + (rl >> 1)) + (rl & 1)] = w;
  }
  __syncthreads();
  float2* Z = fft_lines(A, B, LS, kXPairs, Rx, stw, -1);
  // split the two spectra: X_k = (Z_k + conj Z_-k)/2, Y_k = -i (Z_k - conj Z_-k)/2
  float2* out = R.spec + (size_t)comp * nrows * mxh;
  for (int e = threadIdx.x; e < kXPairs * mxh; e += blockDim.x) {
    int l = e / mxh, k = e - l * mxh;
    int Rw = row0 + 2 * l;
    if (Rw >= nrows) continue;
    float2 zk = Z[k * LS + l];
    float2 zm = Z[((mx - k) % mx) * LS + l];
    float2 X = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    float2 Y = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    out[(size_t)Rw * mxh + k] = X;
    if (Rw + 1 < nrows) out[(size_t)(Rw + 1) * mxh + k] = Y;
  }
}

// Complex transform along y of the half spectrum, in place.
// blockIdx.z = 3 * instance + component.
template <bool ONE>
__global__ void __launch_bounds__(kFftThreads)
    k_yfft(FSL_KARGS, Radices Ry, const float2* __restrict__ tw, int dir) {
  FSL_REP_AT(blockIdx.z / 3);
  extern __shared__ float2 smem[];
  const int my = P.my, mxh = P.mxh;
  const int LS = kYTile;
  float2* A = smem;
  float2* B = A + my * LS;
  float2* stw = B + my * LS;
  const int kx0 = blockIdx.x * kYTile, z = blockIdx.y, comp = blockIdx.z % 3;
  for (int t = threadIdx.x; t < my; t += blockDim.x) stw[t] = tw[t];
  float2* base = R.spec + ((size_t)comp * P.mz + z) * (size_t)my * mxh;
  for (int e = threadIdx.x; e < my * kYTile; e += blockDim.x) {
    int l = e % kYTile, y = e / kYTile;
    int kx = kx0 + l;
    A[y * LS + l] = kx < mxh ? base[(size_t)y * mxh + kx] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* Z = fft_lines(A, B, LS, kYTile, Ry, stw, dir);
  for (int e = threadIdx.x; e < my * kYTile; e += blockDim.x) {
    int l = e % kYTile, y = e / kYTile;
    int kx = kx0 + l;
    if (kx < mxh) base[(size_t)y * mxh + kx] = Z[y * LS + l];
  }
}

// Transform along z, Stokes solve of every mode, inverse transform along z.
// Per mode (src/stokesLimitFunctions.cu:2399-2451 with the shifts of
// src/realToComplex.cu:263-303 and the 1/ncells of :40-59):
//   W'_a = W_a e^{-i pi j_a/m_a};  G2 = |g|^2, g_a = 2/h_a sin(pi j_a/m_a)
//   V'_a = (W'_a - g_a (g.W')/G2) / (eta G2);  v_a = V'_a e^{+i pi j_a/m_a}/nc
//   and v = 0 for the zero mode.  blockIdx.z = instance.
template <bool ONE, int MZ>
__global__ void __launch_bounds__(kFftThreads)
    k_zsolve(FSL_KARGS, Radices Rz, const float2* __restrict__ tw, const float* __restrict__ sx,
             const float* __restrict__ sy, const float* __restrict__ sz,
             const float2* __restrict__ ex, const float2* __restrict__ ey,
             const float2* __restrict__ ez) {
  FSL_REP_AT(blockIdx.z);
  extern __shared__ float2 smem[];
  const int mz = MZ ? MZ : P.mz, my = P.my, mxh = P.mxh;
  constexpr int NLc = 3 * kZTile;
  const int NL = NLc, LS = NL;
  float2* A = smem;
  float2* B = A + mz * LS;
  float2* stw = B + mz * LS;
  const int kx0 = blockIdx.x * kZTile, ky = blockIdx.y;
  for (int t = threadIdx.x; t < mz; t += blockDim.x) stw[t] = tw[t];
  float2* spec = R.spec;
  const size_t cstride = (size_t)mz * my * mxh, zstride = (size_t)my * mxh;
  for (int e = threadIdx.x; e < mz * NL; e += blockDim.x) {
    int lx = e % kZTile, r = e / kZTile;
    int z = r % mz, comp = r / mz;
    int kx = kx0 + lx;
    A[z * LS + comp * kZTile + lx] =
        kx < mxh ? spec[comp * cstride + z * zstride + (size_t)ky * mxh + kx] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* Z = fft_any<MZ, NLc, NLc>(A, B, Rz, stw, -1);
  const float inv_eta = (float)(1.0 / P.eta);
  const float inv_nc = 1.0f / (float)P.nc;
  const float tdx = (float)(2.0 * P.invdx), tdy = (float)(2.0 * P.invdy), tdz = (float)(2.0 * P.invdz);
  for (int e = threadIdx.x; e < mz * kZTile; e += blockDim.x) {
    int lx = e % kZTile, kz = e / kZTile;
    int kx = kx0 + lx;
    if (kx >= mxh) continue;
    float2* p = Z + kz * LS + lx;
    float2 E[3] = {__ldg(ex + kx), __ldg(ey + ky), __ldg(ez + kz)};
    // src/initializePrefactorFourierSpace.cu:48-66: g = 2/h sin(pi j/m)
    float g[3] = {tdx * __ldg(sx + kx), tdy * __ldg(sy + ky), tdz * __ldg(sz + kz)};
    float2 W[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float2 w = p[a * kZTile];
      W[a] = make_float2(w.x * E[a].x + w.y * E[a].y, w.y * E[a].x - w.x * E[a].y);
    }
    float G2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    if (kx == 0 && ky == 0 && kz == 0) {
#pragma unroll
      for (int a = 0; a < 3; ++a) p[a * kZTile] = make_float2(0.f, 0.f);
      continue;
    }
    float invG2 = 1.0f / G2;
    float2 GW = make_float2(g[0] * W[0].x + g[1] * W[1].x + g[2] * W[2].x,
                            g[0] * W[0].y + g[1] * W[1].y + g[2] * W[2].y);
    float fac = inv_eta * invG2 * inv_nc;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float2 V = make_float2((W[a].x - g[a] * GW.x * invG2) * fac, (W[a].y - g[a] * GW.y * invG2) * fac);
      p[a * kZTile] = make_float2(V.x * E[a].x - V.y * E[a].y, V.y * E[a].x + V.x * E[a].y);
    }
  }
  __syncthreads();
  float2* other = (Z == A) ? B : A;
  float2* Y = fft_any<MZ, NLc, NLc>(Z, other, Rz, stw, +1);
  for (int e = threadIdx.x; e < mz * NL; e += blockDim.x) {
    int lx = e % kZTile, r = e / kZTile;
    int z = r % mz, comp = r / mz;
    int kx = kx0 + lx;
    if (kx < mxh) spec[comp * cstride + z * zstride + (size_t)ky * mxh + kx] = Y[z * LS + comp * kZTile + lx];
  }
}

// Complex-to-real along x: Z_k = X_k + i Y_k (k <= mx/2) and its Hermitian
// completion conj X_{m-k} + i conj Y_{m-k}; the inverse transform gives the
// two real rows as real and imaginary parts.  blockIdx.z = instance.
template <bool ONE>
__global__ void __launch_bounds__(kFftThreads)
    k_xinv(FSL_KARGS, Radices Rx, const float2* __restrict__ tw) {
  FSL_REP_AT(blockIdx.z);
  extern __shared__ float2 smem[];
  const int mx = P.mx, mxh = P.mxh;
  const int LS = kXPairs + 1;
  float2* A = smem;
  float2* B = A + mx * LS;
  float2* stw = B + mx * LS;
  const int comp = blockIdx.y;
  const int nrows = P.my * P.mz;
  const int row0 = blockIdx.x * 2 * kXPairs;
  for (int t = threadIdx.x; t < mx; t += blockDim.x) stw[t] = tw[t];
  const float2* in = R.spec + (size_t)comp * nrows * mxh;
  for (int e = threadIdx.x; e < kXPairs * mxh; e += blockDim.x) {
    int l = e / mxh, k = e - l * mxh;
    int Rw = row0 + 2 * l;
    float2 X = make_float2(0.f, 0.f), Y = make_float2(0.f, 0.f);
    if (Rw < nrows) X = in[(size_t)Rw * mxh + k];
    if (Rw + 1 < nrows) Y = in[(size_t)(Rw + 1) * mxh + k];
    A[k * LS + l] = make_float2(X.x - Y.y, X.y + Y.x);
    int km = mx - k;
    if (k > 0 && km != k && km < mx) A[km * LS + l] = make_float2(X.x + Y.y, Y.x - X.y);
  }
  __syncthreads();
  float2* Z = fft_lines(A, B, LS, kXPairs, Rx, stw, +1);
  const float* Zf = reinterpret_cast<const float*>(Z);
  float* out = R.v + (size_t)comp * P.nc;
  for (int e = threadIdx.x; e < 2 * kXPairs * mx; e += blockDim.x) {
    int rl = e / mx, x = e - rl * mx;
    int Rw = row0 + rl;
    if (Rw < nrows) out[(size_t)Rw * mx + x] = Zf[2 * (x * LS + (rl >> 1)) + (rl & 1)];
  }
}

// ------------------------------------------------------- whole-plane path ---
// One block per (z plane, component, instance) does the whole 2-D transform
// of its plane in shared memory, so a solve is three passes over the fields
// (plane forward, z pencils with the solve, plane inverse) instead of five.
// The plane is kept as its half spectrum P[y][kx]; the 1-D transforms run in
// batches of kPB lines through two small scratch buffers.
constexpr int kPB = 16;

__device__ __forceinline__ int plane_pitch(int mxh) { return mxh | 1; }  // odd: fewer conflicts

template <bool ONE, int MX, int MY>
__global__ void __launch_bounds__(kFftThreads)
    k_plane_fwd(FSL_KARGS, Radices Rx, Radices Ry, const float2* __restrict__ twx,
                const float2* __restrict__ twy) {
  FSL_REP_AT(blockIdx.z);
  extern __shared__ float2 smem[];
  const int mx = MX ? MX : P.mx, my = MY ? MY : P.my, mxh = mx / 2 + 1;
  const int LSP = plane_pitch(mxh);
  constexpr int LS = kPB + 1;
  const int mmax = mx > my ? mx : my;
  float2* Pl = smem;                 // [my][LSP]
  float2* S1 = Pl + my * LSP;        // [mmax][LS]
  float2* S2 = S1 + mmax * LS;       // [mmax][LS]
  float2* tx = S2 + mmax * LS;       // [mx]
  float2* ty = tx + mx;              // [my]
  const int z = blockIdx.x, comp = blockIdx.y;
  for (int t = threadIdx.x; t < mx; t += blockDim.x) tx[t] = twx[t];
  for (int t = threadIdx.x; t < my; t += blockDim.x) ty[t] = twy[t];
  const float* W = R.wbuf + (size_t)comp * P.nc + (size_t)z * my * mx;
  const int npairs = (my + 1) / 2;
  // x: real rows (2p, 2p+1) as one complex line, kPB pairs at a time
  for (int p0 = 0; p0 < npairs; p0 += kPB) {
    float* S1f = reinterpret_cast<float*>(S1);
    for (int e = threadIdx.x; e < 2 * kPB * mx; e += blockDim.x) {
      int rl = e / mx, x = e - rl * mx;
      int y = 2 * p0 + rl;
      float w = (y < my && p0 + (rl >> 1) < npairs) ? W[(size_t)y * mx + x] : 0.0f;
      S1f[2 * (x * LS + (rl >> 1)) + (rl & 1)] = w;
    }
    __syncthreads();
    float2* Z = fft_any<MX, kPB, LS>(S1, S2, Rx, tx, -1);
    for (int e = threadIdx.x; e < kPB * mxh; e += blockDim.x) {
      int l = e / mxh, k = e - l * mxh;
      int y = 2 * (p0 + l);
      if (y >= my) continue;
      float2 zk = Z[k * LS + l];
      float2 zm = Z[((mx - k) % mx) * LS + l];
      Pl[y * LSP + k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
      if (y + 1 < my) Pl[(y + 1) * LSP + k] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    }
    __syncthreads();
  }
  // y: kPB columns at a time, written straight to the spectrum
  float2* out = R.spec + ((size_t)comp * P.mz + z) * (size_t)my * mxh;
  for (int k0 = 0; k0 < mxh; k0 += kPB) {
    for (int e = threadIdx.x; e < my * kPB; e += blockDim.x) {
      int l = e % kPB, y = e / kPB;
      int k = k0 + l;
      S1[y * LS + l] = k < mxh ? Pl[y * LSP + k] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* Z = fft_any<MY, kPB, LS>(S1, S2, Ry, ty, -1);
    for (int e = threadIdx.x; e < my * kPB; e += blockDim.x) {
      int l = e % kPB, y = e / kPB;
      int k = k0 + l;
      if (k < mxh) out[(size_t)y * mxh + k] = Z[y * LS + l];
    }
    __syncthreads();
  }
}

template <bool ONE, int MX, int MY>
__global__ void __launch_bounds__(kFftThreads)
    k_plane_inv(FSL_KARGS, Radices Rx, Radices Ry, const float2* __restrict__ twx,
                const float2* __restrict__ twy) {
  FSL_REP_AT(blockIdx.z);
  extern __shared__ float2 smem[];
  const int mx = MX ? MX : P.mx, my = MY ? MY : P.my, mxh = mx / 2 + 1;
  const int LSP = plane_pitch(mxh);
  constexpr int LS = kPB + 1;
  const int mmax = mx > my ? mx : my;
  float2* Pl = smem;
  float2* S1 = Pl + my * LSP;
  float2* S2 = S1 + mmax * LS;
  float2* tx = S2 + mmax * LS;
  float2* ty = tx + mx;
  const int z = blockIdx.x, comp = blockIdx.y;
  for (int t = threadIdx.x; t < mx; t += blockDim.x) tx[t] = twx[t];
  for (int t = threadIdx.x; t < my; t += blockDim.x) ty[t] = twy[t];
  const float2* in = R.spec + ((size_t)comp * P.mz + z) * (size_t)my * mxh;
  // y: inverse transform of kPB columns at a time into the plane buffer
  for (int k0 = 0; k0 < mxh; k0 += kPB) {
    for (int e = threadIdx.x; e < my * kPB; e += blockDim.x) {
      int l = e % kPB, y = e / kPB;
      int k = k0 + l;
      S1[y * LS + l] = k < mxh ? in[(size_t)y * mxh + k] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* Z = fft_any<MY, kPB, LS>(S1, S2, Ry, ty, +1);
    for (int e = threadIdx.x; e < my * kPB; e += blockDim.x) {
      int l = e % kPB, y = e / kPB;
      int k = k0 + l;
      if (k < mxh) Pl[y * LSP + k] = Z[y * LS + l];
    }
    __syncthreads();
  }
  // x: complex-to-real, two rows per complex line
  const int npairs = (my + 1) / 2;
  float* out = R.v + (size_t)comp * P.nc + (size_t)z * my * mx;
  for (int p0 = 0; p0 < npairs; p0 += kPB) {
    for (int e = threadIdx.x; e < kPB * mxh; e += blockDim.x) {
      int l = e / mxh, k = e - l * mxh;
      int y = 2 * (p0 + l);
      float2 X = make_float2(0.f, 0.f), Y = make_float2(0.f, 0.f);
      if (y < my) X = Pl[y * LSP + k];
      if (y + 1 < my) Y = Pl[(y + 1) * LSP + k];
      S1[k * LS + l] = make_float2(X.x - Y.y, X.y + Y.x);
      int km = mx - k;
      if (k > 0 && km != k && km < mx) S1[km * LS + l] = make_float2(X.x + Y.y, Y.x - X.y);
    }
    __syncthreads();
    float2* Z = fft_any<MX, kPB, LS>(S1, S2, Rx, tx, +1);
    const float* Zf = reinterpret_cast<const float*>(Z);
    for (int e = threadIdx.x; e < 2 * kPB * mx; e += blockDim.x) {
      int rl = e / mx, x = e - rl * mx;
      int y = 2 * p0 + rl;
      if (y < my) out[(size_t)y * mx + x] = Zf[2 * (x * LS + (rl >> 1)) + (rl & 1)];
    }
    __syncthreads();
  }
}

#include "fsl_bulk.cuh"
#include "fsl_fft_reg.cuh"
#include "fsl_fft_lines.cuh"
#include "fsl_fft_v.cuh"

// ------------------------------------------------------------ host side ---
static void use_pcand(FftPlan* fp, int i) {
  const FftPlan::PCand& c = fp->pc[i];
  fp->plane_fwd_r[0] = c.fwd[0];
  fp->plane_fwd_r[1] = c.fwd[1];
  fp->plane_inv_r[0] = c.inv[0];
  fp->plane_inv_r[1] = c.inv[1];
  fp->plane_pb = c.pb;
  fp->plane_threads = c.threads;
  fp->smem_plane_r = c.smem;
}

// One planes-per-block candidate of the register plane passes.
template <int N, int R, int T, int PB>
static void add_pcand(FftPlan* fp) {
  if (fp->npc >= kMaxPCand) return;
  FftPlan::PCand& c = fp->pc[fp->npc++];
  c.fwd[0] = k_plane_fwd_r<false, N, R, T, PB>;
  c.fwd[1] = k_plane_fwd_r<true, N, R, T, PB>;
  c.inv[0] = k_plane_inv_r<false, N, R, T, PB>;
  c.inv[1] = k_plane_inv_r<true, N, R, T, PB>;
  c.pb = PB;
  c.threads = PB * (N / 2) * T;
  c.smem = sizeof(float2) * (N + (size_t)PB * plane_buf<N, R, T>());
}

// The register plane passes of edge N (N = R x T), with planes-per-block
// candidates PB, PBS... (the first is the default), and the five-pass
// line kernels of the same shape.
template <int N, int R, int T, int PB, int... PBS>
static void pick_plane_r(FftPlan* fp) {
  add_pcand<N, R, T, PB>(fp);
  (add_pcand<N, R, T, PBS>(fp), ...);
  if constexpr (T > 1 && 32 % T == 0) {
    fp->line_xf[0] = k_fft_xf<false, N, R, T>;
    fp->line_xf[1] = k_fft_xf<true, N, R, T>;
    fp->line_yf[0] = k_fft_y<false, N, R, T, -1>;
    fp->line_yf[1] = k_fft_y<true, N, R, T, -1>;
    fp->line_yi[0] = k_fft_y<false, N, R, T, +1>;
    fp->line_yi[1] = k_fft_y<true, N, R, T, +1>;
    fp->line_xi[0] = k_fft_xi<false, N, R, T>;
    fp->line_xi[1] = k_fft_xi<true, N, R, T>;
    fp->line_lw = 32 / T;
    fp->smem_lines = sizeof(float2) * (N + (size_t)kLineWarps * (32 / T) * LineGeom<R, T>::LS);
  }
  if constexpr (N == 128 && R == 16 && T == 8 && PB == 1 && sizeof...(PBS) == 0) {
    // the conflict-free layout of the same arithmetic (fsl_fft_v.cuh);
    // FLUAMSL_PLANE_V=0 keeps the generic kernels, for comparison
    const char* e = getenv("FLUAMSL_PLANE_V");
    if (!(e && e[0] == '0')) {
      FftPlan::PCand& c = fp->pc[0];
      c.fwd[0] = k_plane_fwd_v<false>;
      c.fwd[1] = k_plane_fwd_v<true>;
      c.inv[0] = k_plane_inv_v<false>;
      c.inv[1] = k_plane_inv_v<true>;
      c.smem = sizeof(float2) * (size_t)kVSmem;
    }
  }
  use_pcand(fp, 0);
}

// FLUAMSL_PLANE_CAND=i fixes the planes-per-block candidate i of the
// register plane passes (0: the default; past the last: the last) instead
// of letting fft_autotune time them (-1)
static int pcand_env() {
  static const int v = [] {
    const char* e = getenv("FLUAMSL_PLANE_CAND");
    return e && *e ? std::max(0, atoi(e)) : -1;
  }();
  return v;
}

// FLUAMSL_FFT_SCHEDULE=plane or =lines fixes the transform schedule of the
// register path (0: picked by fft_autotune, 1: plane kernels, 2: five passes)
static int sched_env() {
  static const int v = [] {
    const char* e = getenv("FLUAMSL_FFT_SCHEDULE");
    if (!e) return 0;
    if (!strcmp(e, "plane")) return 1;
    if (!strcmp(e, "lines")) return 2;
    return 0;
  }();
  return v;
}

static void use_zcand(FftPlan* fp, int i) {
  const FftPlan::ZCand& c = fp->zc[i];
  fp->zsolve_r[0] = c.k[0];
  fp->zsolve_r[1] = c.k[1];
  fp->z_kx = c.kx;
  fp->z_ky = c.ky;
  fp->z_threads = c.threads;
  fp->smem_z_r = c.smem;
}

template <int MZ, int R, int T, int KX, int KY>
static void pick_z_r(FftPlan* fp) {
  if (fp->nzc >= kMaxZCand) return;
  FftPlan::ZCand& c = fp->zc[fp->nzc++];
  c.k[0] = k_zsolve_r<false, MZ, R, T, KX, KY>;
  c.k[1] = k_zsolve_r<true, MZ, R, T, KX, KY>;
  c.kx = KX;
  c.ky = KY;
  c.threads = 3 * KX * KY * T;
  c.smem = sizeof(float2) * (MZ + (size_t)3 * KX * KY * LineGeom<R, T>::LS);
  if (fp->nzc == 1) use_zcand(fp, 0);
}

// Register-pass shapes per edge: N = R x T; planes per block; z tiles.
static void pick_register_kernels(const Params& P, FftPlan* fp) {
  if (P.mx == P.my) {
    switch (P.mx) {
      case 16: pick_plane_r<16, 16, 1, 16, 8, 32>(fp); break;
      case 24: pick_plane_r<24, 24, 1, 16, 8, 32>(fp); break;
      case 32: pick_plane_r<32, 16, 2, 4, 2, 8>(fp); break;
      case 40: pick_plane_r<40, 8, 5, 4>(fp); break;
      case 48: pick_plane_r<48, 12, 4, 2, 1, 4>(fp); break;
      case 56: pick_plane_r<56, 8, 7, 2>(fp); break;
      case 64: pick_plane_r<64, 16, 4, 2, 1, 4>(fp); break;
      case 72: pick_plane_r<72, 12, 6, 1>(fp); break;
      case 80: pick_plane_r<80, 20, 4, 1>(fp); break;
      case 88: pick_plane_r<88, 8, 11, 1>(fp); break;
      case 96: pick_plane_r<96, 24, 4, 1, 2>(fp); break;
      case 128: pick_plane_r<128, 16, 8, 1>(fp); break;
      default: break;
    }
  }
  switch (P.mz) {
    case 16: pick_z_r<16, 16, 1, 9, 8>(fp); break;
    case 24: pick_z_r<24, 24, 1, 13, 8>(fp); break;
    case 32:
      pick_z_r<32, 16, 2, 17, 4>(fp);
      pick_z_r<32, 16, 2, 9, 8>(fp);
      break;
    case 40: pick_z_r<40, 8, 5, 21, 2>(fp); break;
    case 48:
      pick_z_r<48, 12, 4, 25, 1>(fp);
      pick_z_r<48, 12, 4, 13, 2>(fp);
      break;
    case 56: pick_z_r<56, 8, 7, 29, 1>(fp); break;
    case 64:
      pick_z_r<64, 16, 4, 33, 1>(fp);
      pick_z_r<64, 16, 4, 17, 2>(fp);
      pick_z_r<64, 16, 4, 8, 4>(fp);
      break;
    case 72: pick_z_r<72, 12, 6, 19, 1>(fp); break;
    case 80: pick_z_r<80, 20, 4, 21, 1>(fp); break;
    case 88: pick_z_r<88, 8, 11, 9, 1>(fp); break;
    case 96:
      pick_z_r<96, 24, 4, 25, 1>(fp);
      pick_z_r<96, 24, 4, 13, 2>(fp);
      break;
    case 128:
      pick_z_r<128, 16, 8, 8, 2>(fp);
      pick_z_r<128, 16, 8, 13, 1>(fp);
      pick_z_r<128, 16, 8, 4, 2>(fp);
      pick_z_r<128, 16, 8, 4, 1>(fp);
      pick_z_r<128, 16, 8, 2, 2>(fp);
      break;
    case 256:
      pick_z_r<256, 16, 16, 8, 1>(fp);
      pick_z_r<256, 16, 16, 4, 2>(fp);
      break;
    default: break;
  }
}
template <int M>
static void pick_cubic(FftPlan* fp) {
  fp->plane_fwd[0] = k_plane_fwd<false, M, M>;
  fp->plane_fwd[1] = k_plane_fwd<true, M, M>;
  fp->plane_inv[0] = k_plane_inv<false, M, M>;
  fp->plane_inv[1] = k_plane_inv<true, M, M>;
}

template <int M>
static void pick_z(FftPlan* fp) {
  fp->zsolve[0] = k_zsolve<false, M>;
  fp->zsolve[1] = k_zsolve<true, M>;
}

static void pick_kernels(const Params& P, FftPlan* fp) {
  pick_cubic<0>(fp);
  if (P.mx == P.my) {
    switch (P.mx) {
      case 16: pick_cubic<16>(fp); break;
      case 24: pick_cubic<24>(fp); break;
      case 32: pick_cubic<32>(fp); break;
      case 48: pick_cubic<48>(fp); break;
      case 64: pick_cubic<64>(fp); break;
      case 96: pick_cubic<96>(fp); break;
      case 128: pick_cubic<128>(fp); break;
      default: break;
    }
  }
  switch (P.mz) {
    case 16: pick_z<16>(fp); break;
    case 24: pick_z<24>(fp); break;
    case 32: pick_z<32>(fp); break;
    case 48: pick_z<48>(fp); break;
    case 64: pick_z<64>(fp); break;
    case 96: pick_z<96>(fp); break;
    case 128: pick_z<128>(fp); break;
    case 256: pick_z<256>(fp); break;
    default: pick_z<0>(fp); break;
  }
}

static bool upload_table(const std::vector<float2>& h, float2** d) {
  if (cudaMalloc(d, sizeof(float2) * h.size()) != cudaSuccess) return false;
  return cudaMemcpy(*d, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice) == cudaSuccess;
}
static bool upload_table(const std::vector<float>& h, float** d) {
  if (cudaMalloc(d, sizeof(float) * h.size()) != cudaSuccess) return false;
  return cudaMemcpy(*d, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice) == cudaSuccess;
}

FftPlan* fft_plan_create(const Params& P) {
  FftPlan* fp = new FftPlan();
  if (!factorize(P.mx, fp->rx) || !factorize(P.my, fp->ry) || !factorize(P.mz, fp->rz)) {
    delete fp;
    return nullptr;
  }
  // small-DFT coefficient tables (idempotent)
  float2 w5[5], w7[7], w11[11];
  for (int t = 0; t < 5; ++t) w5[t] = make_float2((float)cos(2 * M_PI * t / 5), (float)-sin(2 * M_PI * t / 5));
  for (int t = 0; t < 7; ++t) w7[t] = make_float2((float)cos(2 * M_PI * t / 7), (float)-sin(2 * M_PI * t / 7));
  for (int t = 0; t < 11; ++t) w11[t] = make_float2((float)cos(2 * M_PI * t / 11), (float)-sin(2 * M_PI * t / 11));
  cudaMemcpyToSymbol(c_w5, w5, sizeof(w5));
  cudaMemcpyToSymbol(c_w7, w7, sizeof(w7));
  cudaMemcpyToSymbol(c_w11, w11, sizeof(w11));
  {
    static float2 rwt[kMaxRegR + 1][kMaxRegR];
    for (int R = 1; R <= kMaxRegR; ++R)
      for (int j = 0; j < kMaxRegR; ++j)
        rwt[R][j] = make_float2((float)cos(2 * M_PI * j / R), (float)-sin(2 * M_PI * j / R));
    cudaMemcpyToSymbol(c_rw, rwt, sizeof(rwt));
  }

  const int m[3] = {P.mx, P.my, P.mz};
  float2** tws[3] = {&fp->twx, &fp->twy, &fp->twz};
  float** ss[3] = {&fp->sx, &fp->sy, &fp->sz};
  float2** es[3] = {&fp->ex, &fp->ey, &fp->ez};
  double pi = 4. * atan(1.);
  for (int a = 0; a < 3; ++a) {
    std::vector<float2> tw(m[a]), e(m[a]);
    std::vector<float> sn(m[a]);
    for (int t = 0; t < m[a]; ++t) {
      double ang = 2.0 * pi * (double)t / (double)m[a];
      tw[t] = make_float2((float)cos(ang), (float)-sin(ang));
      // src/initializePrefactorFourierSpace.cu:48-66 (times 2/h in the kernel)
      sn[t] = (float)sin(pi * t / double(m[a]));
      e[t] = make_float2((float)cos(pi * t / double(m[a])), (float)sin(pi * t / double(m[a])));
    }
    if (!upload_table(tw, tws[a]) || !upload_table(sn, ss[a]) || !upload_table(e, es[a])) {
      fft_plan_destroy(fp);
      return nullptr;
    }
  }
  fp->smem_x = sizeof(float2) * (2 * (size_t)P.mx * (kXPairs + 1) + P.mx);
  fp->smem_y = sizeof(float2) * (2 * (size_t)P.my * kYTile + P.my);
  fp->smem_z = sizeof(float2) * (2 * (size_t)P.mz * 3 * kZTile + P.mz);
  // Every kernel's dynamic limit is raised to the most the device allows
  // beside the kernel's own static shared memory (the batched forms hold a
  // copy of their instance there), not to this plan's need: kernels with
  // runtime sizes are shared by plans of different sizes, and a larger limit
  // costs nothing.  A kernel whose need exceeds its limit is not used.
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      optin <= 0)
    optin = 227 * 1024;
  auto allow = [&](const void* f, size_t need) {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, f) != cudaSuccess) return false;
    const int most = optin - (int)a.sharedSizeBytes;
    if (most <= 0 || need > (size_t)most) return false;
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, most) == cudaSuccess;
  };
  pick_kernels(P, fp);
  bool ok = true;
  for (int v = 0; v < 2; ++v) {
    ok = ok && allow((const void*)(v ? k_xfwd<true> : k_xfwd<false>), fp->smem_x);
    ok = ok && allow((const void*)(v ? k_xinv<true> : k_xinv<false>), fp->smem_x);
    ok = ok && allow((const void*)(v ? k_yfft<true> : k_yfft<false>), fp->smem_y);
    ok = ok && allow((const void*)fp->zsolve[v], fp->smem_z);
  }
  if (!ok) {
    cudaGetLastError();
    fft_plan_destroy(fp);
    return nullptr;
  }
  {
    int mmax = P.mx > P.my ? P.mx : P.my;
    int lsp = P.mxh | 1;
    fp->smem_plane = sizeof(float2) * ((size_t)P.my * lsp + 2 * (size_t)mmax * (kPB + 1) + P.mx + P.my);
    fp->use_plane = true;
    for (int v = 0; v < 2; ++v)
      fp->use_plane = fp->use_plane && allow((const void*)fp->plane_fwd[v], fp->smem_plane) &&
                      allow((const void*)fp->plane_inv[v], fp->smem_plane);
  }
  pick_register_kernels(P, fp);
  {
    // keep the planes-per-block candidates whose shared memory fits
    int kept = 0;
    for (int i = 0; i < fp->npc; ++i) {
      const FftPlan::PCand& c = fp->pc[i];
      bool fits = true;
      for (int v = 0; v < 2; ++v)
        fits = fits && allow((const void*)c.fwd[v], c.smem) && allow((const void*)c.inv[v], c.smem);
      if (fits) fp->pc[kept++] = c;
    }
    fp->npc = kept;
    if (kept) {
      use_pcand(fp, pcand_env() < 0 ? 0 : std::min(pcand_env(), kept - 1));
    } else {
      fp->plane_fwd_r[0] = fp->plane_fwd_r[1] = nullptr;
      fp->plane_inv_r[0] = fp->plane_inv_r[1] = nullptr;
    }
  }
  for (int v = 0; v < 2; ++v) {
    if (fp->line_xf[0] &&
        !(allow((const void*)fp->line_xf[v], fp->smem_lines) && allow((const void*)fp->line_yf[v], fp->smem_lines) &&
          allow((const void*)fp->line_yi[v], fp->smem_lines) && allow((const void*)fp->line_xi[v], fp->smem_lines)))
      fp->line_xf[0] = fp->line_xf[1] = nullptr;
  }
  {
    // keep the z candidates whose shared memory fits
    int kept = 0;
    for (int i = 0; i < fp->nzc; ++i)
      if (allow((const void*)fp->zc[i].k[0], fp->zc[i].smem) && allow((const void*)fp->zc[i].k[1], fp->zc[i].smem))
        fp->zc[kept++] = fp->zc[i];
    fp->nzc = kept;
    if (kept) use_zcand(fp, 0);
    else fp->zsolve_r[0] = fp->zsolve_r[1] = nullptr;
  }
  // the five-pass schedule needs the register plane shapes (the same
  // packing) and the register z pass; it starts as the default where it
  // exists, and fft_autotune keeps whichever is faster
  if (!fp->plane_fwd_r[0] || !fp->zsolve_r[0]) fp->line_xf[0] = fp->line_xf[1] = nullptr;
  fp->use_lines = fp->line_xf[0] != nullptr && sched_env() != 1;
  cudaGetLastError();
  // the tables went up with plain copies on the default stream; the step
  // runs on other streams
  if (cudaDeviceSynchronize() != cudaSuccess) {
    fft_plan_destroy(fp);
    return nullptr;
  }
  fp->ok = true;
  return fp;
}

void fft_plan_destroy(FftPlan* fp) {
  if (!fp) return;
  cudaFree(fp->twx);
  cudaFree(fp->twy);
  cudaFree(fp->twz);
  cudaFree(fp->sx);
  cudaFree(fp->sy);
  cudaFree(fp->sz);
  cudaFree(fp->ex);
  cudaFree(fp->ey);
  cudaFree(fp->ez);
  delete fp;
}

static void zsolve(const Batch& B, const FftPlan* fp, dim3 gz, cudaStream_t s) {
  if (fp->zsolve_r[0]) {
    dim3 g((B.mxh + fp->z_kx - 1) / fp->z_kx, (B.my + fp->z_ky - 1) / fp->z_ky, B.nrep);
    if (B.one)
      fsl_launch(fp->zsolve_r[1], g, fp->z_threads, fp->smem_z_r, s, RepSrc{}, *B.one, fp->twz, fp->sx,
                 fp->sy, fp->sz, fp->ex, fp->ey, fp->ez);
    else
      fsl_launch(fp->zsolve_r[0], g, fp->z_threads, fp->smem_z_r, s, B.src(), Rep{}, fp->twz, fp->sx,
                 fp->sy, fp->sz, fp->ex, fp->ey, fp->ez);
    return;
  }
  if (B.one)
    fp->zsolve[1]<<<gz, kFftThreads, fp->smem_z, s>>>(RepSrc{}, *B.one, fp->rz, fp->twz, fp->sx, fp->sy,
                                                     fp->sz, fp->ex, fp->ey, fp->ez);
  else
    fp->zsolve[0]<<<gz, kFftThreads, fp->smem_z, s>>>(B.src(), Rep{}, fp->rz, fp->twz, fp->sx, fp->sy,
                                                     fp->sz, fp->ex, fp->ey, fp->ez);
}

// The register path's transforms and solve with the plan's schedule: the
// plane kernels (3 launches) or the five passes of warp tasks.
static void reg_transform(const Batch& B, const FftPlan* fp, cudaStream_t s, Prof& pr) {
  const int nrep = B.nrep;
  if (fp->use_lines) {
    const long lines = 3L * B.mz * (B.mx / 2);
    const long per_block = (long)kLineWarps * fp->line_lw;
    const dim3 g((unsigned)((lines + per_block - 1) / per_block), 1, nrep);
    const int tb = kLineWarps * 32;
    const size_t sm = fp->smem_lines;
    auto go = [&](void (*const* k)(RepSrc, Rep, const float2*)) {
      if (B.one) fsl_launch(k[1], g, tb, sm, s, RepSrc{}, *B.one, fp->twx);
      else fsl_launch(k[0], g, tb, sm, s, B.src(), Rep{}, fp->twx);
    };
    pr.mark(s, "fft_x");
    go(fp->line_xf);
    pr.mark(s, "fft_y");
    go(fp->line_yf);
    pr.mark(s, "zsolve");
    zsolve(B, fp, dim3(1), s);
    pr.mark(s, "fft_y");
    go(fp->line_yi);
    pr.mark(s, "fft_x");
    go(fp->line_xi);
    pr.count(5);
    return;
  }
  dim3 gp((3 * B.mz + fp->plane_pb - 1) / fp->plane_pb, 1, nrep);
  const int tb = fp->plane_threads;
  pr.mark(s, "plane_fwd");
  if (B.one)
    fsl_launch(fp->plane_fwd_r[1], gp, tb, fp->smem_plane_r, s, RepSrc{}, *B.one, fp->twx);
  else
    fsl_launch(fp->plane_fwd_r[0], gp, tb, fp->smem_plane_r, s, B.src(), Rep{}, fp->twx);
  pr.mark(s, "zsolve");
  zsolve(B, fp, dim3((B.mxh + kZTile - 1) / kZTile, B.my, nrep), s);
  pr.mark(s, "plane_inv");
  if (B.one)
    fsl_launch(fp->plane_inv_r[1], gp, tb, fp->smem_plane_r, s, RepSrc{}, *B.one, fp->twx);
  else
    fsl_launch(fp->plane_inv_r[0], gp, tb, fp->smem_plane_r, s, B.src(), Rep{}, fp->twx);
  pr.count(3);
}

// Times the z-pass tile candidates on the class's own spectra (an in-place
// transform and solve of whatever they hold: the next step rewrites them) and
// keeps the fastest; then, where the edge has both, the plane schedule
// against the five-pass one (on the class's W, spectra and velocity buffers,
// which the step rewrites before reading).  Every candidate computes the
// same bits, so the choice does not change results.  Once per plan, outside
// graph capture.
void fft_autotune(FftPlan* fp, const Batch& B, cudaStream_t s) {
  if (!fp || fp->tuned) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
  fp->tuned = true;
  if (B.nrep == 0 || B.prec == PREC_F64 || !fp->zsolve_r[0]) return;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    cudaGetLastError();
    return;
  }
  // three rounds over the candidates in turn (clock ramp-up and cold caches
  // hit every candidate alike), five launches each, the fastest round kept
  for (int i = 0; i < fp->nzc; ++i) fp->zc_us[i] = 1e30f;
  for (int round = 0; round < 3 && fp->nzc > 1; ++round)
    for (int i = 0; i < fp->nzc; ++i) {
      use_zcand(fp, i);
      zsolve(B, fp, dim3(1), s);  // warm-up
      cudaEventRecord(e0, s);
      for (int r = 0; r < 5; ++r) zsolve(B, fp, dim3(1), s);
      cudaEventRecord(e1, s);
      float ms = 0.f;
      if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) ms = 1e9f;
      fp->zc_us[i] = std::min(fp->zc_us[i], ms * 1000.f / 5.f);
    }
  int best = 0;
  for (int i = 1; i < fp->nzc; ++i)
    if (fp->zc_us[i] < fp->zc_us[best]) best = i;
  use_zcand(fp, best);
  // planes per block of the plane schedule: the whole transform timed per
  // candidate, as the z tiles
  if (fp->npc > 1 && pcand_env() < 0 && sched_env() != 2) {
    const bool lines = fp->use_lines;
    fp->use_lines = false;
    Prof none;
    for (int i = 0; i < fp->npc; ++i) fp->pc_us[i] = 1e30f;
    for (int round = 0; round < 3; ++round)
      for (int i = 0; i < fp->npc; ++i) {
        use_pcand(fp, i);
        reg_transform(B, fp, s, none);  // warm-up
        cudaEventRecord(e0, s);
        for (int r = 0; r < 5; ++r) reg_transform(B, fp, s, none);
        cudaEventRecord(e1, s);
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) ms = 1e9f;
        fp->pc_us[i] = std::min(fp->pc_us[i], ms * 1000.f / 5.f);
      }
    int pbest = 0;
    for (int i = 1; i < fp->npc; ++i)
      if (fp->pc_us[i] < fp->pc_us[pbest]) pbest = i;
    use_pcand(fp, pbest);
    fp->use_lines = lines;
  }
  if (fp->line_xf[0] && sched_env() == 0) {
    Prof none;
    fp->sched_us[0] = fp->sched_us[1] = 1e30f;
    for (int round = 0; round < 3; ++round)
      for (int sc = 0; sc < 2; ++sc) {
        fp->use_lines = sc == 1;
        reg_transform(B, fp, s, none);  // warm-up
        cudaEventRecord(e0, s);
        for (int r = 0; r < 5; ++r) reg_transform(B, fp, s, none);
        cudaEventRecord(e1, s);
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) ms = 1e9f;
        fp->sched_us[sc] = std::min(fp->sched_us[sc], ms * 1000.f / 5.f);
      }
    fp->use_lines = fp->sched_us[1] < fp->sched_us[0];
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGetLastError();
}

void fft_tuning(const FftPlan* fp, FftTuning& out) {
  out = FftTuning{};
  out.schedule = -1;
  if (!fp) return;
  out.tuned = fp->tuned ? 1 : 0;
  if (fp->plane_fwd_r[0]) out.schedule = fp->use_lines ? 1 : 0;
  out.z_kx = fp->z_kx;
  out.z_ky = fp->z_ky;
  out.z_threads = fp->z_threads;
  out.nz = std::min(fp->nzc, 8);
  for (int i = 0; i < out.nz; ++i) out.z_us[i] = fp->zc_us[i] < 1e29f ? fp->zc_us[i] : 0.f;
  for (int k = 0; k < 2; ++k) out.sched_us[k] = fp->sched_us[k] < 1e29f ? fp->sched_us[k] : 0.f;
  out.plane_pb = fp->plane_fwd_r[0] ? fp->plane_pb : 0;
  out.npc = std::min(fp->npc, 4);
  for (int i = 0; i < out.npc; ++i) out.plane_us[i] = fp->pc_us[i] < 1e29f ? fp->pc_us[i] : 0.f;
}

void launch_field_clear(const Batch& B, cudaStream_t s) {
  if (B.nrep == 0) return;
  const long cap = (148L * 8 + B.nrep - 1) / B.nrep;
  long blocks = ((long)3 * B.nc * 8 / 16 + 255) / 256;
  if (blocks > cap) blocks = cap < 1 ? 1 : cap;
  FSL_GO(k_field_clear, dim3((unsigned)blocks, B.nrep), 256, 0, s, B);
}

void launch_solve(const Batch& B, FftPlan* fp, int nsets, double nfac, int w_given, cudaStream_t s,
                  Prof* prof, cudaEvent_t w_built) {
  if (B.prec == PREC_F64) return launch_solve64(B, nsets, nfac, s, prof);
  Prof dummy;
  Prof& pr = prof ? *prof : dummy;
  const int nrep = B.nrep;
  if (!w_given) {
    // W from the spread field and the noise; clears the spread field
    pr.mark(s, "wbuild");
    int tb = 256;
    long blocks = ((long)B.nc + tb - 1) / tb;
    long cap = (148L * 64 + nrep - 1) / nrep;
    if (blocks > cap) blocks = cap < 1 ? 1 : cap;
    if ((B.mx & 3) == 0) {
      long b4 = ((long)B.nc / 4 + tb - 1) / tb;
      if (b4 > cap) b4 = cap < 1 ? 1 : cap;
      FSL_GO(k_wbuild4, dim3((unsigned)b4, nrep), tb, 0, s, B, nsets, nfac, w_built ? 0 : 1);
    } else {
      FSL_GO(k_wbuild, dim3((unsigned)blocks, nrep), tb, 0, s, B, nsets, nfac, w_built ? 0 : 1);
    }
    pr.count(1);
    if (w_built) cudaEventRecord(w_built, s);
  }
  if (fp->plane_fwd_r[0]) {
    reg_transform(B, fp, s, pr);
    return;
  }
  if (fp->use_plane) {
    dim3 gp(B.mz, 3, nrep);
    pr.mark(s, "plane_fwd");
    if (B.one)
      fp->plane_fwd[1]<<<gp, kFftThreads, fp->smem_plane, s>>>(RepSrc{}, *B.one, fp->rx, fp->ry, fp->twx, fp->twy);
    else
      fp->plane_fwd[0]<<<gp, kFftThreads, fp->smem_plane, s>>>(B.src(), Rep{}, fp->rx, fp->ry, fp->twx, fp->twy);
    dim3 gz((B.mxh + kZTile - 1) / kZTile, B.my, nrep);
    pr.mark(s, "zsolve");
    zsolve(B, fp, gz, s);
    pr.mark(s, "plane_inv");
    if (B.one)
      fp->plane_inv[1]<<<gp, kFftThreads, fp->smem_plane, s>>>(RepSrc{}, *B.one, fp->rx, fp->ry, fp->twx, fp->twy);
    else
      fp->plane_inv[0]<<<gp, kFftThreads, fp->smem_plane, s>>>(B.src(), Rep{}, fp->rx, fp->ry, fp->twx, fp->twy);
    pr.count(3);
    return;
  }
  const int nrows = B.my * B.mz;
  const int npairs = (nrows + 1) / 2;
  dim3 gx((npairs + kXPairs - 1) / kXPairs, 3, nrep);
  pr.mark(s, "xfwd");
  FSL_GO(k_xfwd, gx, kFftThreads, fp->smem_x, s, B, fp->rx, fp->twx);
  dim3 gy((B.mxh + kYTile - 1) / kYTile, B.mz, 3 * nrep);
  pr.mark(s, "yfft");
  FSL_GO(k_yfft, gy, kFftThreads, fp->smem_y, s, B, fp->ry, fp->twy, -1);
  dim3 gz((B.mxh + kZTile - 1) / kZTile, B.my, nrep);
  pr.mark(s, "zsolve");
  zsolve(B, fp, gz, s);
  pr.mark(s, "yfft");
  FSL_GO(k_yfft, gy, kFftThreads, fp->smem_y, s, B, fp->ry, fp->twy, +1);
  pr.mark(s, "xinv");
  FSL_GO(k_xinv, gx, kFftThreads, fp->smem_x, s, B, fp->rx, fp->twx);
  pr.count(5);
}

}  // namespace fsl
