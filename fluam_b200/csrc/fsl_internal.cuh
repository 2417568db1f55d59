// fsl_internal.cuh -- shared definitions of the sm_100a Stokes-limit path.
//
// Numerics of the CUDA path (the error against the FP64 oracle is checked by
// the tests for each of these choices):
//   * particle positions, their increments and the cell-index arithmetic are
//     FP64, evaluated with explicitly rounded operations (__dmul_rn, ...), so
//     cell lists and stencil choices are bit-identical to the FP64 oracle;
//   * forces are FP64 (few per step);
//   * spreading accumulates 64-bit fixed point (2^-40) with integer atomics,
//     so the spread field is independent of the order of the atomics and the
//     whole step is bit-reproducible run to run;
//   * kernel weights, the noise, the fields, the FFTs and the spectral
//     multiplier are FP32.
// Two other forms of the fluid side exist for the precision study
// (Params::prec): float atomics instead of the fixed point, and FP64
// everywhere (fsl_fp64.cu).
#pragma once

#include <cstdint>
#include <utility>
#include <cuda_runtime.h>

namespace fsl {

constexpr double kFixedScale = 1099511627776.0;      // 2^40
constexpr double kFixedInv = 1.0 / 1099511627776.0;  // 2^-40
constexpr double kFixedMax = 4611686018427387904.0;  // 2^62
constexpr double kRfdDelta = 0.001;  // src/stokesLimitFunctions.cu:1719
constexpr int kLjTableSize = 4096;   // src/initForcesNonBonded.cu:36

enum { ERR_ANY = 0, ERR_BITS = 1 };
// Params::prec, the values of FSL_PRECISION_* (include/fluamsl.h)
enum { PREC_FIXED = 0, PREC_FLOAT = 1, PREC_F64 = 2 };

// The ten round keys of Philox4x32-10 for one seed (philox_keys).
struct PhiloxKeys {
  uint32_t k0[10], k1[10];
};

// Everything a kernel needs about one instance, passed by value.
struct Params {
  // fluid grid
  int mx, my, mz, mxh;  // mxh = mx/2 + 1 (half spectrum along x)
  int nc;
  double lx, ly, lz, dx, dy, dz;
  double invdx, invdy, invdz, invlx, invly, invlz, dV;
  // non-bonded neighbour grid, m = max(3, int(L / rc))
  int mnx, mny, mnz, mN;
  double invdnx, invdny, invdnz;  // m / L
  // particles and physics
  int np;
  int kernel;  // 3 or 4
  int pair, nonbonded, rfd, bonded;
  int scheme;  // FSL_SCHEME_* (0 midpoint, 1 first order, 2 quasi2D, 3 stokesLimit2D)
  int prec;    // FSL_PRECISION_* (0 fixed point, 1 float atomics, 2 FP64)
  int observe; // FP64 observables accumulated at the end of every step
  // pair forces from a Verlet list (soft repulsion): pairs within
  // rc + skin at the reference positions qref, rebuilt when a particle has
  // moved more than skin / 2 since; nolist: no pair forces, no cell list
  int verlet, nolist;
  double skin, vl_cut2, vl_half2;  // skin, (rc + skin)^2, (skin / 2)^2
  int has_extra;
  double cutoff, cutoff2, invcut2, soft_eps;
  double eta, kT, dt, extra_mob, fact1, fact2, fact4;
  uint64_t seed;
  PhiloxKeys keys;   // the round keys of seed (set with it on the host)
  uint64_t noise_n;  // 12 nc + 9 np; quasi-2D family 4 (nc + mx + my) + 2 np nDrift
  // quasi-2D family: Gaussian variance, stencil half-width, stochastic
  // prefactor, options
  double q2_var, q2_fact1, q2_kc, q2_lw, q2_shear;
  int q2_kw, q2_rfd, q2_pc, q2_ndrift;
  // incompressible scheme: fluid density
  double rho;
};

// noise count of an instance of P with np particles
__host__ __device__ inline uint64_t noise_count(const Params& P, int np) {
  if (P.scheme == 4) return (uint64_t)6 * P.nc;
  if (P.scheme >= 2)
    return (uint64_t)4 * ((uint64_t)P.nc + P.mx + P.my) + (uint64_t)2 * np * P.q2_ndrift;
  return (uint64_t)12 * P.nc + (uint64_t)9 * np;
}

// ---------------------------------------------------------------- Philox ---
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): multipliers
// 0xD2511F53 / 0xCD9E8D57, key increments 0x9E3779B9 / 0xBB67AE85.
__host__ __device__ inline uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
#endif
}

__host__ __device__ inline uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0 = mulhi32(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    uint32_t hi1 = mulhi32(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// The same rounds with the key schedule computed beforehand (the round keys
// depend on the seed only; Params::keys holds the instance's).
__host__ __device__ inline PhiloxKeys philox_keys(uint64_t seed) {
  PhiloxKeys K;
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  for (int r = 0; r < 10; ++r) {
    K.k0[r] = k0;
    K.k1[r] = k1;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return K;
}
__host__ __device__ inline uint4 philox4x32_10(uint4 c, const PhiloxKeys& K) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0 = mulhi32(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    uint32_t hi1 = mulhi32(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ K.k0[r], lo1, hi0 ^ c.w ^ K.k1[r], lo0);
  }
  return c;
}

// The four normal deviates of one Philox output r.  Word w becomes the
// uniform (2 (w >> 9) + 1) 2^-24 in (0,1), exact in FP32; Box-Muller on the
// pairs (u0,u1) and (u2,u3).
__device__ inline float4 philox_box_muller(uint4 r) {
  const float s24 = 5.9604644775390625e-08f;  // 2^-24
  float u0 = (float)(2u * (r.x >> 9) + 1u) * s24;
  float u1 = (float)(2u * (r.y >> 9) + 1u) * s24;
  float u2 = (float)(2u * (r.z >> 9) + 1u) * s24;
  float u3 = (float)(2u * (r.w >> 9) + 1u) * s24;
  float ra = sqrtf(-2.0f * logf(u0));
  float rb = sqrtf(-2.0f * logf(u2));
  // the angle 2 pi u taken as 2 pi (u - 1/2) + pi, within [-pi, pi] where the
  // hardware sine and cosine are accurate to about 2^-21 (u - 1/2 is exact);
  // the radius keeps the accurate logarithm
  float sa, ca, sb, cb;
  __sincosf(6.28318530717958647692f * (u1 - 0.5f), &sa, &ca);
  __sincosf(6.28318530717958647692f * (u3 - 0.5f), &sb, &cb);
  return make_float4(-ra * ca, -ra * sa, -rb * cb, -rb * sb);
}

// philox_normal4 with the key schedule K of the seed (philox_keys)
__device__ inline float4 philox_normal4(const PhiloxKeys& K, uint64_t t, uint64_t b) {
  const uint4 c = make_uint4((uint32_t)b, (uint32_t)(b >> 32), (uint32_t)t, (uint32_t)(t >> 32));
  return philox_box_muller(philox4x32_10(c, K));
}

// The four normal deviates with noise indices 4b .. 4b+3 of draw t
// (philox_box_muller of the Philox output of counter (b, t) keyed by seed).
__device__ inline float4 philox_normal4(uint64_t seed, uint64_t t, uint64_t b) {
  const uint4 c = make_uint4((uint32_t)b, (uint32_t)(b >> 32), (uint32_t)t, (uint32_t)(t >> 32));
  return philox_box_muller(philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32)));
}

// ------------------------------------------------------------ W of a cell ---
// The solve's right-hand side W of one cell: the spread field's sum over the
// cell volume (fixed point, scale = 2^-40 / dV, or the FP32 sum of the
// float-atomic form, fscale = 1 / dV) plus fac times the noise divergence,
// with one FP32 FMA for the noise term.  Every W builder (the W kernels and
// the tiled spread) rounds alike.
__device__ __forceinline__ float w_fixed(long long g, float scale, float fac, float d) {
  return __fmaf_rn(fac, d, (float)((double)g * (double)scale));
}
__device__ __forceinline__ float w_float(float g, float fscale, float fac, float d) {
  return __fmaf_rn(fac, d, __fmul_rn(g, fscale));
}

// --------------------------------------------------- exact cell indices ---
__device__ __forceinline__ double dsgn(double r) { return (double)((r > 0) - (r < 0)); }

// r - int(r/L + sign(r)/2) L, src/stokesLimitFunctions.cu:41-49
__device__ __forceinline__ double minimage(double r, double invL, double L) {
  double t = __dadd_rn(__dmul_rn(r, invL), __dmul_rn(0.5, dsgn(r)));
  return __dsub_rn(r, __dmul_rn((double)(int)t, L));
}

// int(r m/L + m/2) % m of a wrapped coordinate.  For finite coordinates
// within the box this is the reference's formula; any other input (NaN, a
// coordinate beyond the int range) still lands in [0, m), so no index
// derived from it can leave its array, and the caller flags the value.
__device__ __forceinline__ int cellidx(double r, double invd, int m) {
  int j = (int)__dadd_rn(__dmul_rn(r, invd), __dmul_rn(0.5, (double)m));
  // a wrapped coordinate gives j in [0, m] (m only at r = L/2): one
  // comparison; anything else takes the general remainder
  if (j == m) return 0;
  if ((unsigned)j > (unsigned)m) {
    j %= m;
    j = j < 0 ? j + m : j;
  }
  return j;
}

// (j + k) mod m for j in [0, m), -1 <= k <= 2 and m >= 3 (stencil offsets)
__device__ __forceinline__ int wrap_add(int j, int k, int m) {
  int y = j + k;
  y += y < 0 ? m : 0;
  y -= y >= m ? m : 0;
  return y;
}

__device__ __forceinline__ int nb_cell(const Params& P, double x, double y, double z) {
  int jx = cellidx(minimage(x, P.invlx, P.lx), P.invdnx, P.mnx);
  int jy = cellidx(minimage(y, P.invly, P.ly), P.invdny, P.mny);
  int jz = cellidx(minimage(z, P.invlz, P.lz), P.invdnz, P.mnz);
  return jx + jy * P.mnx + jz * P.mnx * P.mny;
}

// minimage for |r| < 1.5 L (a difference of two wrapped coordinates): the
// same n = int(r/L + sign(r)/2) in {-1, 0, 1}, found by comparisons instead
// of float-to-integer conversions.
__device__ __forceinline__ double minimage_near(double r, double invL, double L) {
  const double t = __dadd_rn(__dmul_rn(r, invL), copysign(0.5, r));
  const double n = t >= 1.0 ? 1.0 : (t <= -1.0 ? -1.0 : 0.0);
  return __dsub_rn(r, __dmul_rn(n, L));
}

// ------------------------------------------------------- Peskin kernels ---
// 3-point kernel, src/deltaGPU.cu:57-68 (argument = distance / h)
__device__ __forceinline__ float delta3f(float x) {
  x = fabsf(x);
  if (x > 1.5f) return 0.0f;
  if (x < 0.5f) return (1.0f + sqrtf(1.0f - 3.0f * x * x)) * (1.0f / 3.0f);
  float y = 1.0f - x;
  return (5.0f - 3.0f * x - sqrtf(fmaxf(1.0f - 3.0f * y * y, 0.0f))) * (1.0f / 6.0f);
}

// 4-point kernel (Peskin, Acta Numerica 2002), the 3-D extension of the
// fractional form of src/deltaGPU.cu:44-53.
__device__ __forceinline__ float delta4f(float x) {
  x = fabsf(x);
  if (x >= 2.0f) return 0.0f;
  if (x <= 1.0f) return (3.0f - 2.0f * x + sqrtf(1.0f + 4.0f * x - 4.0f * x * x)) * 0.125f;
  return (5.0f - 2.0f * x - sqrtf(fmaxf(-7.0f + 12.0f * x - 4.0f * x * x, 0.0f))) * 0.125f;
}

// Node k (0..n-1) of the stencil of field component comp in dimension d:
// grid index j and its weight.  Nodes of component comp in dimension d sit at
// (j + 1/2) h - L/2, plus h/2 when d == comp.  posc picks the nodes, posw sets
// the weight (they differ only in the reference's RFD quirk).
__device__ __forceinline__ void stencil_node(const Params& P, int d, int comp, double posc,
                                             double posw, int k, int& j, float& w) {
  const int m = d == 0 ? P.mx : (d == 1 ? P.my : P.mz);
  const double h = d == 0 ? P.dx : (d == 1 ? P.dy : P.dz);
  const double invd = d == 0 ? P.invdx : (d == 1 ? P.invdy : P.invdz);
  const double L = d == 0 ? P.lx : (d == 1 ? P.ly : P.lz);
  const double invL = d == 0 ? P.invlx : (d == 1 ? P.invly : P.invlz);
  const double off = (d == comp) ? __dmul_rn(0.5, h) : 0.0;
  if (P.kernel == 3) {
    double r = minimage(__dsub_rn(posc, off), invL, L);
    int jc = cellidx(r, invd, m);
    j = wrap_add(jc, k - 1, m);
    double node = ((double)j + 0.5) * h - 0.5 * L;
    double rr = minimage((posw - node) - off, invL, L);
    w = delta3f((float)(rr * invd));
  } else {
    double r = minimage(__dsub_rn(__dsub_rn(posc, off), __dmul_rn(0.5, h)), invL, L);
    int jb = cellidx(r, invd, m);
    j = wrap_add(jb, k - 1, m);
    double node = ((double)j + 0.5) * h - 0.5 * L + off;
    double rr = minimage(posw - node, invL, L);
    w = delta4f((float)(rr * invd));
  }
}

// First node index of the stencil in dimension d, for the cell-centre
// (face == 0) or the face (face == 1) node family; the index arithmetic of
// stencil_node.
__device__ __forceinline__ int stencil_base(const Params& P, int d, int face, double posc) {
  const int m = d == 0 ? P.mx : (d == 1 ? P.my : P.mz);
  const double h = d == 0 ? P.dx : (d == 1 ? P.dy : P.dz);
  const double invd = d == 0 ? P.invdx : (d == 1 ? P.invdy : P.invdz);
  const double L = d == 0 ? P.lx : (d == 1 ? P.ly : P.lz);
  const double invL = d == 0 ? P.invlx : (d == 1 ? P.invly : P.invlz);
  const double off = face ? __dmul_rn(0.5, h) : 0.0;
  double r = P.kernel == 3 ? __dsub_rn(posc, off) : __dsub_rn(__dsub_rn(posc, off), __dmul_rn(0.5, h));
  return cellidx(minimage(r, invL, L), invd, m);
}

// Warp-shared stencil of one particle for all three components.  Per
// dimension d there are two node families: cell centres (components with
// comp != d) and faces (comp == d); with n nodes each that is 6n values,
// lane (f * 3 + d) * n + k computing family f, dimension d, node k.  Every
// lane calls this; the result stays in the computing lane and is read with
// stencil_get.
struct WarpStencil {
  int j;
  float w;
};

__device__ __forceinline__ WarpStencil warp_stencil(const Params& P, const double posc[3],
                                                    const double posw[3], int lane) {
  WarpStencil s{0, 0.0f};
  const int n = P.kernel;
  if (lane < 6 * n) {
    int k = lane % n, fd = lane / n;
    int f = fd / 3, d = fd - 3 * f;
    // selects, not posc[d]: a runtime index would put the arrays on the stack
    const double pc = d == 0 ? posc[0] : (d == 1 ? posc[1] : posc[2]);
    const double pw = d == 0 ? posw[0] : (d == 1 ? posw[1] : posw[2]);
    // family f = 1 is the face family of dimension d: use comp = d
    stencil_node(P, d, f == 1 ? d : (d + 1) % 3, pc, pw, k, s.j, s.w);
  }
  return s;
}

// node k of dimension d for component comp, from the lanes of warp_stencil
__device__ __forceinline__ void stencil_get(const WarpStencil& s, int n, int comp, int d, int k,
                                            int& j, float& w) {
  int src = ((comp == d ? 3 : 0) + d) * n + k;
  j = __shfl_sync(0xffffffffu, s.j, src);
  w = __shfl_sync(0xffffffffu, s.w, src);
}

__device__ __forceinline__ void set_err(int* err, int bit) {
  atomicOr(&err[ERR_BITS], bit);
  err[ERR_ANY] = 1;
}

// ---------------------------------------------------- stress divergence ---
// Noise terms of W for component comp at cell i (x,y,z) for one stress
// sample d (src/stokesLimitFunctions.cu:2323-2367): the divergence of the
// stochastic stress with diagonals at cell centres and off-diagonals on edges.
__device__ __forceinline__ float stress_div(const Params& P, const float* __restrict__ d, int comp,
                                            int x, int y, int z, int i, float a1x, float a1y,
                                            float a1z, float a4x, float a4y, float a4z) {
  const size_t nc = (size_t)P.nc;
  const int mx = P.mx, my = P.my, mz = P.mz;
  int xm = x == 0 ? mx - 1 : x - 1, xp = x == mx - 1 ? 0 : x + 1;
  int ym = y == 0 ? my - 1 : y - 1, yp = y == my - 1 ? 0 : y + 1;
  int zm = z == 0 ? mz - 1 : z - 1, zp = z == mz - 1 ? 0 : z + 1;
  int rowyz = mx * (y + my * z);
  if (comp == 0) {
    int v3 = xp + rowyz, v1 = x + mx * (ym + my * z), v0 = x + mx * (y + my * zm);
    return a1x * (__ldg(d + v3) - __ldg(d + i)) + a4y * (__ldg(d + nc + i) - __ldg(d + nc + v1)) +
           a4z * (__ldg(d + 2 * nc + i) - __ldg(d + 2 * nc + v0));
  } else if (comp == 1) {
    int v4 = x + mx * (yp + my * z), v2 = xm + rowyz, v0 = x + mx * (y + my * zm);
    return a1y * (__ldg(d + 3 * nc + v4) - __ldg(d + 3 * nc + i)) +
           a4x * (__ldg(d + nc + i) - __ldg(d + nc + v2)) +
           a4z * (__ldg(d + 4 * nc + i) - __ldg(d + 4 * nc + v0));
  } else {
    int v5 = x + mx * (y + my * zp), v2 = xm + rowyz, v1 = x + mx * (ym + my * z);
    return a1z * (__ldg(d + 5 * nc + v5) - __ldg(d + 5 * nc + i)) +
           a4x * (__ldg(d + 2 * nc + i) - __ldg(d + 2 * nc + v2)) +
           a4y * (__ldg(d + 4 * nc + i) - __ldg(d + 4 * nc + v1));
  }
}

// Four consecutive x cells of a row for one stress sample d: the x, y, z
// neighbours as 16-byte rows (aligned: the sample's base is a multiple of 4
// floats; otherwise four scalar loads) plus the two x-edge scalars.
__device__ __forceinline__ float4 ld_row4(const float* __restrict__ p, bool aligned) {
  if (aligned) return __ldg(reinterpret_cast<const float4*>(p));
  return make_float4(__ldg(p), __ldg(p + 1), __ldg(p + 2), __ldg(p + 3));
}

// w[comp][c] += the stress divergence of cells x0 .. x0+3 (the arithmetic of
// stress_div, four cells at a time).
__device__ __forceinline__ void stress_div4(const Params& P, const float* __restrict__ d,
                                            bool aligned, int x0, int y, int z, size_t i0,
                                            float a1x, float a1y, float a1z, float a4x,
                                            float a4y, float a4z, float (&w)[3][4]) {
  const size_t nc = (size_t)P.nc;
  const int mx = P.mx, my = P.my, mz = P.mz;
  const size_t row = i0 - x0;  // first cell of the row
  const long dym = (y == 0 ? (long)(my - 1) * mx : -(long)mx);
  const long dyp = (y == my - 1 ? -(long)(my - 1) * mx : (long)mx);
  const long dzm = (z == 0 ? (long)(mz - 1) * my * mx : -(long)my * mx);
  const long dzp = (z == mz - 1 ? -(long)(mz - 1) * my * mx : (long)my * mx);
  const int xl = x0 == 0 ? mx - 1 : x0 - 1, xr = x0 + 4 == mx ? 0 : x0 + 4;
  const float4 r0 = ld_row4(d + i0, aligned);
  const float e0 = __ldg(d + row + xr);
  const float4 r1 = ld_row4(d + nc + i0, aligned), r1ym = ld_row4(d + nc + i0 + dym, aligned);
  const float e1 = __ldg(d + nc + row + xl);
  const float4 r2 = ld_row4(d + 2 * nc + i0, aligned), r2zm = ld_row4(d + 2 * nc + i0 + dzm, aligned);
  const float e2 = __ldg(d + 2 * nc + row + xl);
  const float4 r3 = ld_row4(d + 3 * nc + i0, aligned), r3yp = ld_row4(d + 3 * nc + i0 + dyp, aligned);
  const float4 r4 = ld_row4(d + 4 * nc + i0, aligned), r4zm = ld_row4(d + 4 * nc + i0 + dzm, aligned),
               r4ym = ld_row4(d + 4 * nc + i0 + dym, aligned);
  const float4 r5 = ld_row4(d + 5 * nc + i0, aligned), r5zp = ld_row4(d + 5 * nc + i0 + dzp, aligned);
  const float d0[5] = {r0.x, r0.y, r0.z, r0.w, e0};          // d0[x .. x+4]
  const float d1[5] = {e1, r1.x, r1.y, r1.z, r1.w};          // d1[x-1 .. x+3]
  const float d2[5] = {e2, r2.x, r2.y, r2.z, r2.w};          // d2[x-1 .. x+3]
  const float d1ym[4] = {r1ym.x, r1ym.y, r1ym.z, r1ym.w}, d2zm[4] = {r2zm.x, r2zm.y, r2zm.z, r2zm.w};
  const float d3[4] = {r3.x, r3.y, r3.z, r3.w}, d3yp[4] = {r3yp.x, r3yp.y, r3yp.z, r3yp.w};
  const float d4[4] = {r4.x, r4.y, r4.z, r4.w}, d4zm[4] = {r4zm.x, r4zm.y, r4zm.z, r4zm.w},
              d4ym[4] = {r4ym.x, r4ym.y, r4ym.z, r4ym.w};
  const float d5[4] = {r5.x, r5.y, r5.z, r5.w}, d5zp[4] = {r5zp.x, r5zp.y, r5zp.z, r5zp.w};
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    w[0][c] += a1x * (d0[c + 1] - d0[c]) + a4y * (d1[c + 1] - d1ym[c]) + a4z * (d2[c + 1] - d2zm[c]);
    w[1][c] += a1y * (d3yp[c] - d3[c]) + a4x * (d1[c + 1] - d1[c]) + a4z * (d4[c] - d4zm[c]);
    w[2][c] += a1z * (d5zp[c] - d5[c]) + a4x * (d2[c + 1] - d2[c]) + a4y * (d4[c] - d4ym[c]);
  }
}

}  // namespace fsl

// ------------------------------------------------- host-side launchers ---
// Declared here, defined in the .cu files; all enqueue on `s`.
namespace fsl {

// Sets the message fsl_last_error() returns on this thread; returns code.
int set_last_error(int code, const char* msg);

// Stage timer: mark(name) records an event on the stream; the interval up to
// the next mark is charged to `name` (nullptr closes the last interval).
// Off by default; when on, the marks are captured into the step's graph too.
struct Prof {
  static constexpr int kMax = 64;
  bool on = false;
  cudaEvent_t ev[kMax] = {};
  const char* name[kMax] = {};
  int used = 0;
  int launches = 0;  // kernels of this library enqueued in the current step
  void mark(cudaStream_t s, const char* n) {
    if (!on || used >= kMax) return;
    if (!ev[used]) cudaEventCreate(&ev[used]);
    // External under stream capture, so that the record becomes an
    // event-record node of the graph (a plain record would only express a
    // dependency); the flag is refused outside capture (the eager first step
    // of an instance, or steps without graphs), where a plain record does
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusActive)
      cudaEventRecordWithFlags(ev[used], s, cudaEventRecordExternal);
    else
      cudaEventRecord(ev[used], s);
    name[used++] = n;
  }
  void count(int k) { launches += k; }
};
// One instance of the step: its parameters and device buffers.  A kernel
// launch serves a batch of instances of one size class (same grid and
// neighbour-grid extents, same kernel width).  A single instance is a batch
// of one and is passed to its kernels by value.
struct Rep {
  Params P;
  int active;  // 0: unused slot, every kernel returns at once
  double *q, *qp, *F;
  int *cell_of, *cnt, *start, *fill, *tmp, *sorted, *bsum;
  int *bpp_cnt, *bpp_off, *bpp_idx;
  double *bpp_k, *bpp_r0;
  int *bfp_cnt, *bfp_off;
  double *bfp_k, *bfp_r0, *bfp_xyz;
  float* ljtab;
  float* noise;
  // the 3-D Stokes schemes: D1 = div(Sigma_1) | D12 = div(Sigma_1 + Sigma_2),
  // [3][nc] each (k_div), read by the W build
  float* ndiv;
  // the midpoint scheme's stencil cache (null elsewhere): planes A, B, C of
  // 4 np lanes each (lane e 4 + a of particle e), the quad_nodes of that
  // lane as written by the last spread (QuadLane packing)
  uint4* stc;
  unsigned long long* grid;
  float2* spec;
  float* v;
  float* wbuf;
  double* u;  // interpolated velocities of the component entry point
  double* qw;  // positions wrapped into the box by the last cell-list build
  double* ws;  // the same in cell-list order
  // the cell list of the second build of a step (at q^{n+1/2}), so that the
  // list at q^n stays readable: start, sorted, ws of build 1 (null when the
  // scheme builds one list per step; build 1 then writes the fields above)
  int* start1;
  int* sorted1;
  double* ws1;
  // FP64 form only (null otherwise): noise, field, complex spectrum
  double* noise64;
  double* v64;
  double2* z64;
  int* err;
  uint64_t* t;
  // observables: reference positions q0 [3][np], accumulators (kObsSlots
  // doubles, the fsl_observables fields in order after the step count),
  // per-block partial sums and the ticket of the last block
  double* q0;
  double* obs;
  double* obs_part;
  unsigned* obs_ticket;
  // Verlet list: per particle count and kVlCap neighbour slots ([slot][np]),
  // reference positions, and the rebuild word vl_flag: [0], [1] the step
  // (counter + 1) at whose force evaluation at q (0) or q^{n+1/2} (1) the
  // list must be rebuilt; [2] 1: rebuild at the next evaluation, 2: cell
  // list requested by an entry point, 3: cell mode (a particle had more
  // than kVlCap neighbours: the pair forces come from the cell list of every
  // evaluation until the positions are set again)
  int* vl_cnt;
  int* vl_idx;
  double* qref;
  uint64_t* vl_flag;
  // grid barrier of the single-launch list build (count, generation)
  unsigned* bar;
};
constexpr int kCoopMaxBlocks = 1024;
constexpr int kVlCap = 64;
constexpr int kObsVals = 10;      // msd, displacement[3], force[3], momentum[3]
constexpr int kObsSlots = 16;     // steps, msd, msd_sum, disp[3], force[3], mom[3], mom_sum[3]
constexpr int kObsMaxBlocks = 148;

// The cell list of build `which` (0: at q^n, 1: at q^{n+1/2}).
struct CellList {
  const int* start;
  const int* sorted;
  const double* ws;
};
__device__ __forceinline__ CellList cell_list(const Rep& R, int which) {
  if (which && R.start1) return CellList{R.start1, R.sorted1, R.ws1};
  return CellList{R.start, R.sorted, R.ws};
}

// Whether the list-building kernels of force evaluation `which` run: always
// for the cell-list path, never without pair forces, and for the Verlet path
// only when the list must be rebuilt.
__device__ __forceinline__ bool list_needed(const Rep& R, int which) {
  if (!R.P.verlet && !R.P.nolist) return true;
  const uint64_t f = R.vl_flag[2];  // 2: requested by a component entry point
  if (f == 2) return true;
  if (R.P.nolist) return false;
  // 3: cell mode (the list overflowed): a cell list at every evaluation
  return f != 0 || R.vl_flag[which] == *R.t + 1;
}

// The quad of this thread in a KIND_T4 launch: particle index e (in the
// instance), lane a in the quad, first lane qb of the quad; returns false
// when the whole warp is past the last particle (uniform per warp).
__device__ __forceinline__ bool quad_of(int blk, int np, long& e, int& a, int& qb) {
  const long t = blk * (long)blockDim.x + threadIdx.x;
  e = t >> 2;
  a = threadIdx.x & 3;
  qb = (threadIdx.x & 31) & ~3;
  return ((t & ~31L) >> 2) < np;
}

// Launch kinds of the particle kernels (256-thread blocks): threads per
// particle 1 (cell list), 8 (forces), 32 (one warp per particle), 4 (one
// quad per particle: spreading and interpolation).
enum { KIND_T1 = 0, KIND_T8 = 1, KIND_T32 = 2, KIND_T4 = 3, NKIND = 4 };
constexpr int kPartThreads = 256;
__host__ __device__ constexpr int kind_threads(int k) { return k == 0 ? 1 : k == 1 ? 8 : k == 2 ? 32 : 4; }
__host__ __device__ constexpr int kind_ppb(int k) { return kPartThreads / kind_threads(k); }

// Where a batched kernel finds its instance: the device table, and for the
// particle kernels the first block of every instance per launch kind,
// boff[kind * (nrep + 1) + r] (a flat grid with no idle blocks for small
// instances).
struct RepSrc {
  const Rep* reps;
  const int* boff;
  int nrep;
};

// Launch shape of a batch: sizes shared by the class and the largest
// per-instance ones.
struct Batch {
  const Rep* reps;  // device table
  const int* boff;  // device block offsets, [NKIND][nrep + 1]
  int nrep;
  int mx, my, mz, mxh, nc, mN, kernel;
  int prec;  // FSL_PRECISION_* of the class
  int max_np;
  uint64_t max_noise_n;
  int tiled;        // spread and W build by launch_spread_w
  int has_vl, has_cl;  // instances on the Verlet path / on the cell-list pair path
  int nblk[NKIND];  // total blocks of each particle launch kind
  const Rep* one;   // host copy of the single instance (nrep == 1), else null
  // list build of a batch of small instances, as the class's tuner picked it
  // (-1: not tuned, the block-per-instance build; 0: the separate kernels;
  // 1: the block-per-instance build)
  int lists_pick = -1;
  RepSrc src() const { return RepSrc{reps, boff, nrep}; }
};

// Instance of a block.  ONE: the launch serves a single instance passed by
// value as a __grid_constant__ parameter, read in place from the parameter
// bank.  Otherwise the block copies its table entry into shared memory.
template <bool ONE>
__device__ __forceinline__ const Rep& rep_copy(const RepSrc& src, const Rep& one, int idx, Rep& sh) {
  if constexpr (ONE) {
    return one;
  } else {
    const int* from = reinterpret_cast<const int*>(src.reps + idx);
    int* to = reinterpret_cast<int*>(&sh);
    for (int k = threadIdx.x; k < (int)(sizeof(Rep) / sizeof(int)); k += blockDim.x) to[k] = __ldg(from + k);
    __syncthreads();
    return sh;
  }
}

// Particle kernels: the instance of this block of the flat grid and the
// block's index within that instance (blk).
template <bool ONE>
__device__ __forceinline__ const Rep& rep_flat(const RepSrc& src, const Rep& one, int kind, int& blk,
                                               Rep& sh) {
  if constexpr (ONE) {
    blk = blockIdx.x;
    return one;
  } else {
    __shared__ int s_r;
    const int* off = src.boff + kind * (src.nrep + 1);
    if (threadIdx.x == 0) {
      // largest r with off[r] <= blockIdx.x (instances without blocks are
      // skipped because their successor starts at the same offset)
      int lo = 0, hi = src.nrep - 1;
      const int b = (int)blockIdx.x;
      while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(off + mid) <= b) lo = mid;
        else hi = mid - 1;
      }
      s_r = lo;
    }
    __syncthreads();
    const int r = s_r;
    blk = (int)blockIdx.x - __ldg(off + r);
    return rep_copy<false>(src, one, r, sh);
  }
}

#define FSL_KARGS const RepSrc src, const __grid_constant__ Rep one

// Programmatic dependent launch.  The kernels that take their instance
// through FSL_REP_AT / FSL_REP_FLAT are launched (fsl_launch) so that their
// blocks may be scheduled while the previous kernel of the stream drains;
// before anything else each block waits until that kernel has completed
// and its writes are visible (griddepcontrol.wait, which returns at once
// for an ordinary launch), then lets the next kernel be scheduled in turn.
// Every kernel of a chain waits before it can complete, so a kernel sees
// the writes of all kernels before it in the stream, not only the last.
__device__ __forceinline__ void fsl_pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

#define FSL_REP_AT(IDX)                                            \
  fsl_pdl_enter();                                                 \
  __shared__ Rep fsl_sh_rep_;                                      \
  const Rep& R = rep_copy<ONE>(src, one, (int)(IDX), fsl_sh_rep_); \
  if (!R.active) return;                                           \
  const Params& P = R.P

#define FSL_REP_FLAT(KIND)                                         \
  fsl_pdl_enter();                                                 \
  __shared__ Rep fsl_sh_rep_;                                      \
  int blk;                                                         \
  const Rep& R = rep_flat<ONE>(src, one, (KIND), blk, fsl_sh_rep_); \
  if (!R.active) return;                                           \
  const Params& P = R.P

// Whether launches carry the programmatic-serialisation attribute
// (FLUAMSL_PDL=0: ordinary launches, for comparison).
bool pdl_enabled();

// Launch of a kernel that enters through FSL_REP_AT / FSL_REP_FLAT, with
// programmatic dependent launch where enabled.  Errors are left for
// cudaPeekAtLastError, as with the <<<>>> syntax.
template <typename... KArgs, typename... Args>
inline void fsl_launch(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// Launch of a kernel template whose first template argument is ONE.
#define FSL_GO(KERN, GRID, BLOCK, SMEM, S, B, ...)                                          \
  do {                                                                                      \
    if ((B).one)                                                                            \
      fsl_launch(KERN<true>, (GRID), (BLOCK), (SMEM), (S), RepSrc{}, *(B).one, ##__VA_ARGS__); \
    else                                                                                    \
      fsl_launch(KERN<false>, (GRID), (BLOCK), (SMEM), (S), (B).src(), Rep{}, ##__VA_ARGS__);  \
  } while (0)
// ... with a second template argument T
#define FSL_GO_T(KERN, T, GRID, BLOCK, SMEM, S, B, ...)                                        \
  do {                                                                                         \
    if ((B).one)                                                                               \
      fsl_launch(KERN<true, T>, (GRID), (BLOCK), (SMEM), (S), RepSrc{}, *(B).one, ##__VA_ARGS__); \
    else                                                                                       \
      fsl_launch(KERN<false, T>, (GRID), (BLOCK), (SMEM), (S), (B).src(), Rep{}, ##__VA_ARGS__);  \
  } while (0)

// Blocks of a particle launch of kind k.
inline unsigned part_blocks(const Batch& B, int k) {
  if (B.one) return (unsigned)(((long)B.max_np * kind_threads(k) + kPartThreads - 1) / kPartThreads);
  return (unsigned)B.nblk[k];
}

// The noise of one step in two parts.  Part 0 draws the normals in the
// reference's layout; for the 3-D Stokes schemes (scheme 0 midpoint, 1 first
// order) it also turns stress sample 1 into its divergence D1 (k_div), and
// part 1 (midpoint only) adds the divergence of sample 2 into D12.  For the
// other schemes part 1 does nothing.
void launch_noise(const Batch& B, cudaStream_t s, int scheme, int part);
void launch_noise_range(const Params& P, uint64_t t, uint64_t first, int64_t count, float* out,
                        cudaStream_t s);
// which = 0: cell list / forces at q, 1: at q^{n+1/2}.  The build leaves the
// count and fill arrays cleared; zero_first clears them (and start, for an
// instance without particles) first, for callers that cannot rely on that.
void launch_cells(const Batch& B, int which, cudaStream_t s, bool zero_first = true);
// vl = false leaves the Verlet-list instances' forces to the spread that
// follows (launch_spread with forces = true)
void launch_forces(const Batch& B, int which, cudaStream_t s, bool vl = true);
// drift = 0: spread F at q (cell-list order when ordered != 0);
// drift = 1: spread F at q^{n+1/2} and the RFD drift at q;
// drift = 2: spread F at q and the RFD drift at q (first-order scheme).
// forces: the Verlet-list instances compute F at the spread's positions in
// the spread kernel (and store it) instead of reading it.  cache: the
// spread stores its quads' nodes and weights in Rep::stc (midpoint scheme)
// for an interpolation at the same positions.
void launch_spread(const Batch& B, int drift, int ordered, cudaStream_t s, bool forces = false,
                   bool cache = false);
// stage 1: q^{n+1/2} = q + dt/2 J(q) v; stage 2: q^{n+1} = q + dt J(q^{n+1/2}) v.
// cached: the nodes come from Rep::stc, written by the spread at the same
// positions (midpoint scheme), instead of being computed again.
void launch_interp_update(const Batch& B, int stage, cudaStream_t s, bool cached = false);
void launch_interp(const Batch& B, cudaStream_t s);  // u = J(q) v
void launch_step_counter(const Batch& B, cudaStream_t s);
// The fixed-point form's spread and W build in one tiled pass (drift as
// launch_spread; nsets, nfac as the W build of launch_solve, which is then
// called with w_given = 1).  tile_eligible: whether a class may use it;
// tile_init sets the kernels' shared-memory limit (once per device).
void tile_init();
bool tile_eligible(const Params& P);
void launch_spread_w(const Batch& B, int drift, int nsets, double nfac, cudaStream_t s);
// The cell list of force evaluation `which` and, for Verlet-list
// instances, the pair list (each only where list_needed says so).
cudaError_t launch_pair_lists(const Batch& B, int which, cudaStream_t s);
// Whether launch_pair_lists builds the lists of this batch in one launch of
// one block per instance: batches of small instances (block_lists_eligible),
// unless the class's tuner picked the separate kernels.
// FLUAMSL_BLOCK_LISTS=0 / =1 fixes the separate kernels / the block build.
bool block_lists_eligible(const Batch& B);
bool block_lists(const Batch& B);
// -1: the tuner decides; 0, 1: fixed by FLUAMSL_BLOCK_LISTS
int block_lists_env();
// Times both list builds of force evaluation 0 of an eligible batch (three
// rounds of three builds each, the fastest round kept) and returns the us
// per build: us[0] the separate kernels, us[1] the block per instance.  A
// build at unchanged positions leaves the lists as they are.
void lists_autotune(const Batch& B, cudaStream_t s, float us[2]);
// The cell-list counters and the single-launch build's barrier cleared
// (after an error, before lists are built again)
void launch_reset_lists(const Rep& r, cudaStream_t s);
// After positions were replaced from the host: flag a Verlet-list rebuild if
// a particle moved more than skin / 2 from its reference position.
void launch_moved_check(const Rep& r, cudaStream_t s);
// FP64 observables of every instance with P.observe (end of a step)
void launch_observe(const Batch& B, cudaStream_t s);
// The FP64 form (fsl_fp64.cu); the launchers above hand a class of that
// form to these.
void launch_noise64(const Batch& B, cudaStream_t s);
void launch_spread64(const Batch& B, int drift, cudaStream_t s);
void launch_interp_update64(const Batch& B, int stage, cudaStream_t s);
void launch_solve64(const Batch& B, int nsets, double nfac, cudaStream_t s, Prof* prof);
// 2-D transforms of two FP64 components (the quasi-2D family)
void launch_fft64_2d(const Batch& B, int dir, cudaStream_t s);
// 3-D transforms of three FP64 components; to_real: the inverse's last pass
// stores Re / nc to Rep::v64 instead of the spectrum
void launch_fft64_3d(const Batch& B, int dir, int to_real, cudaStream_t s);
// The incompressible scheme (fsl_inc.cu)
void launch_inc_w(const Batch& B, int second, cudaStream_t s);
void launch_inc_fourier(const Batch& B, int solve, cudaStream_t s);
void launch_inc_pred(const Batch& B, cudaStream_t s);
void launch_inc_load(const Batch& B, cudaStream_t s);
// The quasi-2D family (fsl_q2d.cu)
void launch_q2_forces(const Batch& B, cudaStream_t s);
void launch_q2_field(const Batch& B, cudaStream_t s, Prof* prof);
void launch_q2_solve(const Batch& B, cudaStream_t s, Prof* prof);
void launch_q2_update(const Batch& B, int stage, cudaStream_t s);

struct FftPlan;  // defined in fsl_fft.cu
FftPlan* fft_plan_create(const Params& P);
void fft_plan_destroy(FftPlan* fp);
// Picks the fastest z-pass tile of the plan's candidates, the fastest
// planes-per-block candidate of the plane passes, then the faster of the
// plane and five-pass transform schedules, on B's buffers (once per plan;
// no-op under stream capture).
void fft_autotune(FftPlan* fp, const Batch& B, cudaStream_t s);
// What the plan's tuner picked and measured (schedule -1: the plan has no
// register path; z tile 0 x 0: no candidates)
struct FftTuning {
  int tuned, schedule, z_kx, z_ky, z_threads, nz;
  float z_us[8], sched_us[2];
  int plane_pb, npc;
  float plane_us[4];
};
void fft_tuning(const FftPlan* fp, FftTuning& out);
// v = solve(W).  W = f + nfac div(stress 1 [+ stress 2 when nsets == 2]) is
// built from the spread field (which is cleared on the way) and the noise
// divergence into Rep::wbuf, unless w_given, in which case Rep::wbuf already
// holds W.  With w_built, the W build leaves the field as it is and records
// w_built after itself: the caller clears the field (launch_field_clear)
// after that event and before the next spread.
void launch_solve(const Batch& B, FftPlan* fp, int nsets, double nfac, int w_given, cudaStream_t s,
                  Prof* prof = nullptr, cudaEvent_t w_built = nullptr);
// Zeroes the spread fields of B's instances (streaming stores).
void launch_field_clear(const Batch& B, cudaStream_t s);
}  // namespace fsl
