// fsl_particles.cu -- particle-side kernels of the Stokes-limit step:
// noise, counting-sort cell list, pair/bonded forces, fixed-point spreading
// (forces and random-finite-difference drift), interpolation + midpoint
// updates.
#include "fsl_internal.cuh"

namespace fsl {

// ------------------------------------------------------------------ noise ---
// The noise array of one draw, in the reference's layout
// (src/runSchemeStokesLimit.cu:86-90, src/randomNumbers.cu:37-40):
// [0,6nc) stress 1 (XX,XY,XZ,YY,YZ,ZZ), [6nc,6nc+3np) RFD vector,
// [6nc+3np,6nc+9np) extra-mobility noises, [6nc+9np,12nc+9np) stress 2.
__global__ void k_noise(uint64_t seed, const uint64_t* __restrict__ t_dev, uint64_t n,
                        float4* __restrict__ out) {
  uint64_t t = *t_dev;
  uint64_t nb = (n + 3) >> 2;
  for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nb;
       b += (uint64_t)gridDim.x * blockDim.x)
    out[b] = philox_normal4(seed, t, b);
}

__global__ void k_noise_range(uint64_t seed, uint64_t t, uint64_t first, int64_t count,
                              float* __restrict__ out) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= count) return;
  uint64_t n = first + (uint64_t)k;
  float4 v = philox_normal4(seed, t, n >> 2);
  int lane = (int)(n & 3);
  out[k] = lane == 0 ? v.x : lane == 1 ? v.y : lane == 2 ? v.z : v.w;
}

void launch_noise(const Params& P, const uint64_t* t_dev, float* out, cudaStream_t s) {
  uint64_t nb = (P.noise_n + 3) / 4;
  int threads = 256;
  int blocks = (int)((nb + threads - 1) / threads);
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_noise<<<blocks, threads, 0, s>>>(P.seed, t_dev, P.noise_n, reinterpret_cast<float4*>(out));
}

void launch_noise_range(const Params& P, uint64_t t, uint64_t first, int64_t count, float* out,
                        cudaStream_t s) {
  if (count <= 0) return;
  k_noise_range<<<(int)((count + 255) / 256), 256, 0, s>>>(P.seed, t, first, count, out);
}

// -------------------------------------------------------------- cell list ---
// Counting sort of the particles by non-bonded cell: count, exclusive scan,
// scatter, then order each cell's particles by index so that the list is
// deterministic (the reference appends with atomics, in arbitrary order:
// src/stokesLimitFunctions.cu:52-57).
__global__ void k_cell_count(Params P, const double* __restrict__ q, int* __restrict__ cell_of,
                             int* __restrict__ cnt, int* __restrict__ err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.np) return;
  double x = q[i], y = q[P.np + i], z = q[2 * P.np + i];
  // a coordinate this large or non-finite means the run has blown up
  const double lim = 1e15;
  if (!(fabs(x) < lim && fabs(y) < lim && fabs(z) < lim)) set_err(err, 2);
  int c = nb_cell(P, x, y, z);
  cell_of[i] = c;
  atomicAdd(&cnt[c], 1);
}

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-local exclusive scan of cnt into start, block totals into bsum.
__global__ void __launch_bounds__(kScanThreads) k_scan_local(const int* __restrict__ cnt, int n,
                                                             int* __restrict__ start,
                                                             int* __restrict__ bsum) {
  __shared__ int warp_tot[kScanThreads / 32];
  int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
  int sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (base + k < n) ? cnt[base + k] : 0;
    sum += v[k];
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int wt = warp_tot[lane];
    int wi = wt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    warp_tot[lane] = wi - wt;  // exclusive
    if (lane == 31) bsum[blockIdx.x] = wi;
  }
  __syncthreads();
  int run = warp_tot[warp] + incl - sum;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) start[base + k] = run;
    run += v[k];
  }
}

// Exclusive scan of the block totals (at most kScanTile of them), in place;
// also writes the grand total to start[n].
__global__ void __launch_bounds__(kScanThreads) k_scan_top(int* __restrict__ bsum, int nb,
                                                           int* __restrict__ start, int n) {
  __shared__ int warp_tot[kScanThreads / 32];
  int base = threadIdx.x * kScanItems;
  int v[kScanItems];
  int sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (base + k < nb) ? bsum[base + k] : 0;
    sum += v[k];
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int wt = warp_tot[lane];
    int wi = wt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    warp_tot[lane] = wi - wt;
    if (lane == 31) start[n] = wi;
  }
  __syncthreads();
  int run = warp_tot[warp] + incl - sum;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < nb) bsum[base + k] = run;
    run += v[k];
  }
}

__global__ void k_scan_add(int* __restrict__ start, int n, const int* __restrict__ bsum) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  start[i] += bsum[i / kScanTile];
}

__global__ void k_cell_scatter(Params P, const int* __restrict__ cell_of,
                               const int* __restrict__ start, int* __restrict__ fill,
                               int* __restrict__ tmp) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.np) return;
  int c = cell_of[i];
  tmp[start[c] + atomicAdd(&fill[c], 1)] = i;
}

// Rank of particle i among the particles of its cell = number of smaller
// indices in the (unordered) bucket; gives the ascending order.
__global__ void k_cell_rank(Params P, const int* __restrict__ cell_of,
                            const int* __restrict__ start, const int* __restrict__ tmp,
                            int* __restrict__ sorted) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.np) return;
  int c = cell_of[i];
  int s = start[c], e = start[c + 1];
  int rank = 0;
  for (int k = s; k < e; ++k) rank += tmp[k] < i;
  sorted[s + rank] = i;
}

void launch_cells(const Params& P, const double* q, int* cell_of, int* cnt, int* start,
                  int* fill, int* tmp, int* sorted, int* bsum, int* err, cudaStream_t s) {
  cudaMemsetAsync(cnt, 0, sizeof(int) * P.mN, s);
  cudaMemsetAsync(fill, 0, sizeof(int) * P.mN, s);
  if (P.np == 0) {
    cudaMemsetAsync(start, 0, sizeof(int) * (P.mN + 1), s);
    return;
  }
  int tb = 256, nbp = (P.np + tb - 1) / tb;
  k_cell_count<<<nbp, tb, 0, s>>>(P, q, cell_of, cnt, err);
  int nblk = (P.mN + kScanTile - 1) / kScanTile;
  k_scan_local<<<nblk, kScanThreads, 0, s>>>(cnt, P.mN, start, bsum);
  k_scan_top<<<1, kScanThreads, 0, s>>>(bsum, nblk, start, P.mN);
  k_scan_add<<<(P.mN + 255) / 256, 256, 0, s>>>(start, P.mN, bsum);
  k_cell_scatter<<<nbp, tb, 0, s>>>(P, cell_of, start, fill, tmp);
  k_cell_rank<<<nbp, tb, 0, s>>>(P, cell_of, start, tmp, sorted);
}

// ----------------------------------------------------------------- forces ---
// Texture-unit linear filtering of a normalised, clamped float table, done in
// software: x_B = x N - 1/2, weight rounded to 8 fractional bits.
__device__ __forceinline__ float tex_linear(const float* __restrict__ T, int N, float x) {
  double xb = (double)x * (double)N - 0.5;
  double fl = floor(xb);
  int i = (int)fl;
  float a = (float)(rint((xb - fl) * 256.0) * (1.0 / 256.0));
  int i0 = min(max(i, 0), N - 1);
  int i1 = min(max(i + 1, 0), N - 1);
  return __fadd_rn(__fmul_rn(1.0f - a, __ldg(T + i0)), __fmul_rn(a, __ldg(T + i1)));
}

// Neighbour-cell order of the reference's pair loop
// (src/stokesLimitFunctions.cu:191-653).
__constant__ signed char c_nb_order[27][3] = {
    {0, 0, 0},   {0, 0, -1},  {0, -1, 0},  {-1, 0, 0},  {1, 0, 0},   {0, 1, 0},
    {0, 0, 1},   {1, 1, 0},   {1, -1, 0},  {1, 0, 1},   {1, 0, -1},  {-1, 1, 0},
    {-1, -1, 0}, {-1, 0, 1},  {-1, 0, -1}, {0, 1, 1},   {0, 1, -1},  {0, -1, 1},
    {0, -1, -1}, {1, 1, 1},   {1, 1, -1},  {1, -1, 1},  {1, -1, -1}, {-1, 1, 1},
    {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};

__device__ __forceinline__ void bond_force(double rx, double ry, double rz, double x, double y,
                                           double z, double k, double r0, double& fx,
                                           double& fy, double& fz) {
  // src/forceBondedGPU.cu:60-75
  if (r0 == 0) {
    fx += -k * (rx - x);
    fy += -k * (ry - y);
    fz += -k * (rz - z);
  } else {
    double r = sqrt((x - rx) * (x - rx) + (y - ry) * (y - ry) + (z - rz) * (z - rz));
    if (r > 0) {
      double a = -k * (1 - r0 / r);
      fx += a * (rx - x);
      fy += a * (ry - y);
      fz += a * (rz - z);
    }
  }
}

__global__ void k_forces(Params P, const double* __restrict__ q, const int* __restrict__ cell_of,
                         const int* __restrict__ start, const int* __restrict__ sorted,
                         const int* __restrict__ bpp_cnt, const int* __restrict__ bpp_off,
                         const int* __restrict__ bpp_idx, const double* __restrict__ bpp_k,
                         const double* __restrict__ bpp_r0, const int* __restrict__ bfp_cnt,
                         const int* __restrict__ bfp_off, const double* __restrict__ bfp_k,
                         const double* __restrict__ bfp_r0, const double* __restrict__ bfp_xyz,
                         const float* __restrict__ ljtab, double* __restrict__ F,
                         int* __restrict__ err) {
  // eight lanes per particle: they share the bonds and the 27 neighbour
  // cells (cells sub, sub+8, ...), then sum their partial forces
  const int sub = threadIdx.x & 7;
  const int ig = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 3);
  const bool active = ig < P.np;  // inactive lanes still join the shuffles
  const int i = active ? ig : 0;
  const int np = P.np;
  double rx = q[i], ry = q[np + i], rz = q[2 * np + i];
  double fx = 0.0, fy = 0.0, fz = 0.0;
  if (P.bonded && active) {
    int nb = bpp_cnt[i], off = bpp_off[i];
    for (int j = sub; j < nb; j += 8) {
      int idx = bpp_idx[off + j];
      bond_force(rx, ry, rz, q[idx], q[np + idx], q[2 * np + idx], bpp_k[off + j],
                 bpp_r0[off + j], fx, fy, fz);
    }
    nb = bfp_cnt[i];
    off = bfp_off[i];
    for (int j = sub; j < nb; j += 8) {
      const double* p = bfp_xyz + 3 * (off + j);
      bond_force(rx, ry, rz, p[0], p[1], p[2], bfp_k[off + j], bfp_r0[off + j], fx, fy, fz);
    }
  }
  if (P.nonbonded && P.pair != 0 && active) {
    int c = cell_of[i];
    int cxy = c % (P.mnx * P.mny);
    int cz = c / (P.mnx * P.mny), cy = cxy / P.mnx, cx = cxy - cy * P.mnx;
    for (int nn = sub; nn < 27; nn += 8) {
      // the 27 cells in z-major order; the summation order only moves the
      // result at the FP64 rounding level
      int ox = cx + nn % 3 - 1, oy = cy + (nn / 3) % 3 - 1, oz = cz + nn / 9 - 1;
      ox += ox < 0 ? P.mnx : (ox >= P.mnx ? -P.mnx : 0);
      oy += oy < 0 ? P.mny : (oy >= P.mny ? -P.mny : 0);
      oz += oz < 0 ? P.mnz : (oz >= P.mnz ? -P.mnz : 0);
      int cc = ox + oy * P.mnx + oz * P.mnx * P.mny;
      int e = start[cc + 1];
      for (int jj = start[cc]; jj < e; ++jj) {
        int j = sorted[jj];
        double rxij = minimage(rx - q[j], P.invlx, P.lx);
        double ryij = minimage(ry - q[np + j], P.invly, P.ly);
        double rzij = minimage(rz - q[2 * np + j], P.invlz, P.lz);
        // no fused multiply-add: r^2 selects the table entry bit-exactly
        double r2 = __dadd_rn(__dadd_rn(__dmul_rn(rxij, rxij), __dmul_rn(ryij, ryij)),
                              __dmul_rn(rzij, rzij));
        double f;
        if (P.pair == 1) {
          f = (double)tex_linear(ljtab, kLjTableSize, (float)(r2 * P.invcut2));
        } else {
          if (j == i || r2 >= P.cutoff2 || r2 == 0.0) continue;
          double r = sqrt(r2);
          f = (2.0 * P.soft_eps / P.cutoff) * (1.0 - r / P.cutoff) / r;
        }
        fx += f * rxij;
        fy += f * ryij;
        fz += f * rzij;
      }
    }
  }
  // fixed butterfly order within the eight lanes: the same sum on every run
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
  }
  if (sub != 0 || !active) return;
  if (!isfinite(fx) || !isfinite(fy) || !isfinite(fz)) set_err(err, 2);
  F[i] = fx;
  F[np + i] = fy;
  F[2 * np + i] = fz;
}

void launch_forces(const Params& P, const double* q, const int* cell_of, const int* start,
                   const int* sorted, const int* bpp_cnt, const int* bpp_off, const int* bpp_idx,
                   const double* bpp_k, const double* bpp_r0, const int* bfp_cnt,
                   const int* bfp_off, const double* bfp_k, const double* bfp_r0,
                   const double* bfp_xyz, const float* ljtab, double* F, int* err,
                   cudaStream_t s) {
  if (P.np == 0) return;
  const int tb = 256, per_block = tb / 8;
  k_forces<<<(P.np + per_block - 1) / per_block, tb, 0, s>>>(P, q, cell_of, start, sorted, bpp_cnt, bpp_off,
                                               bpp_idx, bpp_k, bpp_r0, bfp_cnt, bfp_off, bfp_k,
                                               bfp_r0, bfp_xyz, ljtab, F, err);
}

// ------------------------------------------------------------- spreading ---
// One warp per (entry, component); lane l takes stencil nodes l, l+32, ...
// (x fastest, so a warp's atomics fall on a few 32-byte sectors) and adds
// w * value in 64-bit fixed point to the staggered field of that component.
// Replaces the slot writes of kernelSpreadParticlesForceStokesLimit and
// kernelSpreadParticlesDrift + the gather of addSpreadedForcesStokesLimit
// (src/stokesLimitFunctions.cu:659-1681, 1705-2255); the 1/dV of the gather
// is applied when the field is read back.
//
// Entries [0, nforce) spread F of particle order[e] at qf; entries
// [nforce, nforce + 2 np) spread the RFD drift (kT/delta) sign W_p from
// q + sign (delta/2) W_p, sign + for the first np and - for the second.  In
// reference mode the drift's nodes come from the displaced position and its
// weights from q, as the reference does.
template <int KN>  // kernel width 3 or 4
__device__ __forceinline__ void spread_entry(const Params& P, const double posc[3],
                                             const double posw[3], const double val[3],
                                             unsigned long long* __restrict__ grid, int lane,
                                             bool& sat) {
  constexpr int n = KN, n3 = n * n * n, total = 3 * n3;
  const WarpStencil st = warp_stencil(P, posc, posw, lane);
  constexpr int iters = (total + 31) >> 5;
#pragma unroll
  for (int it = 0; it < iters; ++it) {
    const int id = (it << 5) + lane;
    const bool valid = id < total;
    const int idc = valid ? id : 0;  // every lane takes part in the shuffles
    const int comp = idc / n3, r = idc - comp * n3;
    const int a = r % n, b = (r / n) % n, c = r / (n * n);
    int x, y, z;
    float wx, wy, wz;
    stencil_get(st, n, comp, 0, a, x, wx);
    stencil_get(st, n, comp, 1, b, y, wy);
    stencil_get(st, n, comp, 2, c, z, wz);
    if (!valid) continue;
    const double vc = comp == 0 ? val[0] : (comp == 1 ? val[1] : val[2]);
    double v = (double)(wx * (wy * wz)) * (vc * kFixedScale);
    sat |= !(fabs(v) < kFixedMax);
    long long iv = sat ? 0ll : __double2ll_rn(v);
    if (iv != 0)
      atomicAdd(grid + (size_t)comp * P.nc + x + (size_t)P.mx * (y + (size_t)P.my * z),
                (unsigned long long)iv);
  }
}

// One warp per entry (all three components of one spread of one particle).
template <int KN>
__global__ void k_spread(Params P, int nforce, int drift, const int* __restrict__ order,
                         const double* __restrict__ qf, const double* __restrict__ F,
                         const double* __restrict__ q0, const float* __restrict__ noise,
                         unsigned long long* __restrict__ grid, int* __restrict__ err) {
  const int lane = threadIdx.x & 31;
  const long e = (long)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int np = P.np;
  const long nent = (long)nforce + (drift ? (long)np : 0l);
  if (e >= nent) return;  // uniform per warp
  bool sat = false;
  if (e < nforce) {
    int i = order ? order[e] : (int)e;
    double pos[3] = {qf[i], qf[np + i], qf[2 * np + i]};
    double val[3] = {F[i], F[np + i], F[2 * (size_t)np + i]};
    spread_entry<KN>(P, pos, pos, val, grid, lane, sat);
  } else {
    // both signs of the drift of one particle
    int i = (int)(e - nforce);
    if (order) i = order[i];
    const size_t wbase = (size_t)6 * P.nc;
    double W[3] = {(double)noise[wbase + i], (double)noise[wbase + np + i],
                   (double)noise[wbase + 2 * np + i]};
    double pos[3] = {q0[i], q0[np + i], q0[2 * np + i]};
    double pp[3], pm[3], vp[3], vm[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      pp[d] = pos[d] + 0.5 * kRfdDelta * W[d];
      pm[d] = pos[d] - 0.5 * kRfdDelta * W[d];
      vp[d] = (P.kT / kRfdDelta) * W[d];
      vm[d] = (P.kT / kRfdDelta) * -1 * W[d];
    }
    if (P.rfd != 1) {
      // Reference mode weighs both spreads at q: where both displaced
      // positions pick the same nodes the two fixed-point spreads are exact
      // negatives of each other (same weights, opposite values, symmetric
      // rounding), so they are skipped without changing the result.
      bool same = true;
      if (lane < 6) {
        int f = lane / 3, d = lane - 3 * f;
        same = stencil_base(P, d, f, pp[d]) == stencil_base(P, d, f, pm[d]);
      }
      if (__all_sync(0xffffffffu, same)) return;
      spread_entry<KN>(P, pp, pos, vp, grid, lane, sat);
      spread_entry<KN>(P, pm, pos, vm, grid, lane, sat);
    } else {
      spread_entry<KN>(P, pp, pp, vp, grid, lane, sat);
      spread_entry<KN>(P, pm, pm, vm, grid, lane, sat);
    }
  }
  if (sat) set_err(err, 1);
}

// force spread of all particles (at qf, in the order of the cell list when
// `order` is given) and, with drift != 0, the two RFD spreads at q0
void launch_spread(const Params& P, int drift, const int* order, const double* qf,
                   const double* F, const double* q0, const float* noise,
                   unsigned long long* grid, int* err, cudaStream_t s) {
  if (P.np == 0) return;
  long nent = (long)P.np * (drift ? 2 : 1);
  long threads = nent * 32;
  const int tb = 256;
  unsigned nb = (unsigned)((threads + tb - 1) / tb);
  if (P.kernel == 4)
    k_spread<4><<<nb, tb, 0, s>>>(P, P.np, drift, order, qf, F, q0, noise, grid, err);
  else
    k_spread<3><<<nb, tb, 0, s>>>(P, P.np, drift, order, qf, F, q0, noise, grid, err);
}

// -------------------------------------------------------- interpolation ---
// One warp per particle: lane l reads nodes l, l+32, ... of the three
// components' stencils and the warp sums w v per component in a fixed
// butterfly order (src/stokesLimitFunctions.cu:2616-2642).  Every lane gets
// the three sums.
template <int KN>
__device__ __forceinline__ void interp_particle(const Params& P, const double pos[3],
                                                const float* __restrict__ v, int lane,
                                                float u[3]) {
  constexpr int n = KN, n3 = n * n * n, total = 3 * n3;
  constexpr int iters = (total + 31) >> 5;
  const WarpStencil st = warp_stencil(P, pos, pos, lane);
  // gather every node's address and weight first, then all loads at once
  float wt[iters];
  const float* ad[iters];
#pragma unroll
  for (int it = 0; it < iters; ++it) {
    const int id = (it << 5) + lane;
    const bool valid = id < total;
    const int idc = valid ? id : 0;
    const int comp = idc / n3, r = idc - comp * n3;
    const int a = r % n, b = (r / n) % n, c = r / (n * n);
    int x, y, z;
    float wx, wy, wz;
    stencil_get(st, n, comp, 0, a, x, wx);
    stencil_get(st, n, comp, 1, b, y, wy);
    stencil_get(st, n, comp, 2, c, z, wz);
    wt[it] = valid ? wx * (wy * wz) : 0.0f;
    ad[it] = v + (size_t)comp * P.nc + x + (size_t)P.mx * (y + (size_t)P.my * z);
  }
  float val[iters];
#pragma unroll
  for (int it = 0; it < iters; ++it) val[it] = __ldg(ad[it]);
  float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
#pragma unroll
  for (int it = 0; it < iters; ++it) {
    const int id = (it << 5) + lane;
    const int comp = (id < total ? id : 0) / n3;
    float t = wt[it] * val[it];
    if (comp == 0) s0 += t;
    else if (comp == 1) s1 += t;
    else s2 += t;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  u[0] = s0;
  u[1] = s1;
  u[2] = s2;
}

// stage 1: q^{n+1/2} = q^n + dt/2 J(q^n) v (+ extraMobility terms),
//          src/stokesLimitFunctions.cu:2646-2650
// stage 2: q^{n+1}   = q^n + dt J(q^{n+1/2}) v (+ extraMobility terms),
//          src/stokesLimitFunctions.cu:3676-3681
template <int KN>
__global__ void k_interp_update(Params P, int stage, const double* __restrict__ qpos,
                                const double* __restrict__ q0, const double* __restrict__ F,
                                const float* __restrict__ noise, const float* __restrict__ v,
                                double* __restrict__ qout, int* __restrict__ err) {
  const int lane = threadIdx.x & 31;
  const long t = (long)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  if (t >= P.np) return;  // uniform per warp
  const int i = (int)t;
  const int np = P.np;
  double pos[3] = {qpos[i], qpos[np + i], qpos[2 * np + i]};
  float us[3];
  interp_particle<KN>(P, pos, v, lane, us);
  if (lane >= 3) return;
  const int comp = lane;  // lanes 0, 1, 2 update x, y, z
  const double u = (double)(comp == 0 ? us[0] : (comp == 1 ? us[1] : us[2]));
  size_t k = (size_t)comp * np + i;
  double h = stage == 1 ? 0.5 * P.dt : P.dt;
  double r = q0[k] + h * u;
  if (P.has_extra) {
    size_t nb = (size_t)6 * P.nc + (size_t)(3 + comp) * np + i;
    double xi = (double)noise[nb];
    if (stage == 2) xi += (double)noise[nb + (size_t)3 * np];
    r += h * P.extra_mob * F[k] + P.fact2 * xi;
  }
  if (!isfinite(r)) set_err(err, 2);
  qout[k] = r;
}

template <int KN>
__global__ void k_interp(Params P, const double* __restrict__ qpos, const float* __restrict__ v,
                         double* __restrict__ u) {
  const int lane = threadIdx.x & 31;
  const long t = (long)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  if (t >= P.np) return;  // uniform per warp
  const int i = (int)t;
  const int np = P.np;
  double pos[3] = {qpos[i], qpos[np + i], qpos[2 * np + i]};
  float us[3];
  interp_particle<KN>(P, pos, v, lane, us);
  if (lane < 3) u[(size_t)lane * np + i] = (double)(lane == 0 ? us[0] : (lane == 1 ? us[1] : us[2]));
}

static unsigned warp_blocks(long warps, int tb) {
  return (unsigned)((warps * 32 + tb - 1) / tb);
}

void launch_interp_update(const Params& P, int stage, const double* qpos, const double* q0,
                          const double* F, const float* noise, const float* v, double* qout,
                          int* err, cudaStream_t s) {
  if (P.np == 0) return;
  const int tb = 256;
  if (P.kernel == 4)
    k_interp_update<4><<<warp_blocks(P.np, tb), tb, 0, s>>>(P, stage, qpos, q0, F, noise, v, qout,
                                                            err);
  else
    k_interp_update<3><<<warp_blocks(P.np, tb), tb, 0, s>>>(P, stage, qpos, q0, F, noise, v, qout,
                                                            err);
}

void launch_interp(const Params& P, const double* qpos, const float* v, double* u,
                   cudaStream_t s) {
  if (P.np == 0) return;
  const int tb = 256;
  if (P.kernel == 4)
    k_interp<4><<<warp_blocks(P.np, tb), tb, 0, s>>>(P, qpos, v, u);
  else
    k_interp<3><<<warp_blocks(P.np, tb), tb, 0, s>>>(P, qpos, v, u);
}

__global__ void k_step_counter(uint64_t* t_dev) { *t_dev += 1; }

void launch_step_counter(uint64_t* t_dev, cudaStream_t s) { k_step_counter<<<1, 1, 0, s>>>(t_dev); }

}  // namespace fsl
