// fsl_particles.cu -- particle-side kernels of the Stokes-limit step:
// noise, counting-sort cell list, pair/bonded forces, fixed-point spreading
// (forces and random-finite-difference drift), interpolation + midpoint
// updates.  Every kernel serves a batch of instances (see Rep / Batch in
// fsl_internal.cuh): kernels over cells take the instance from blockIdx.y,
// kernels over particles run a flat grid whose blocks map to instances
// through the block-offset table.  ONE = true compiles the single-instance
// form, whose instance is a by-value parameter.
#include <algorithm>
#include <atomic>
#include <cstdlib>

#include "fsl_internal.cuh"

namespace fsl {

static unsigned blocks_for(long work, int tb) { return (unsigned)((work + tb - 1) / tb); }

// ------------------------------------------------------------------ noise ---
// The noise array of one draw, in the reference's layout
// (src/runSchemeStokesLimit.cu:86-90, src/randomNumbers.cu:37-40):
// [0,6nc) stress 1 (XX,XY,XZ,YY,YZ,ZZ), [6nc,6nc+3np) RFD vector,
// [6nc+3np,6nc+9np) extra-mobility noises, [6nc+9np,12nc+9np) stress 2.
template <bool ONE>
__global__ void k_noise(FSL_KARGS) {
  FSL_REP_AT(blockIdx.y);
  const uint64_t t = *R.t;
  const uint64_t nb = (P.noise_n + 3) >> 2;
  float4* out = reinterpret_cast<float4*>(R.noise);
  for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nb;
       b += (uint64_t)gridDim.x * blockDim.x)
    out[b] = philox_normal4(P.keys, t, b);  // the round keys of P.seed
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

// ------------------------------------------------- stress divergence noise ---
// The 3-D Stokes schemes read the stochastic stress only through its
// divergence (W = f + c div(Sigma), src/stokesLimitFunctions.cu:2281-2378,
// 3922-4069).  k_div turns the drawn stress samples into that divergence on
// the noise's side stream, so the W builds on the step's critical path read
// 3 nc floats instead of 6 nc or 12 nc: set 0 writes D1 = div(Sigma_1) to
// Rep::ndiv, set 1 writes D12 = D1 + div(Sigma_2) after it.  The terms and
// their order are those of stress_div (the W build multiplies D by its
// factor c); one thread per four x cells where mx is a multiple of 4.
template <bool ONE>
__global__ void k_div(FSL_KARGS, int set) {
  FSL_REP_AT(blockIdx.y);
  const size_t nc = (size_t)P.nc;
  const float a1x = (float)P.invdx * (float)P.fact1, a1y = (float)P.invdy * (float)P.fact1,
              a1z = (float)P.invdz * (float)P.fact1;
  const float a4x = (float)P.invdx * (float)P.fact4, a4y = (float)P.invdy * (float)P.fact4,
              a4z = (float)P.invdz * (float)P.fact4;
  const size_t off = set ? (size_t)6 * nc + (size_t)9 * P.np : 0;
  const float* n = R.noise + off;
  float* D = R.ndiv + (set ? 3 * nc : 0);
  if ((P.mx & 3) == 0) {
    const bool aligned = (off & 3) == 0;
    const int gx = P.mx >> 2;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < nc >> 2;
         g += (size_t)gridDim.x * blockDim.x) {
      const int x0 = (int)(g % gx) << 2;
      const int r = (int)(g / gx);
      const int y = r % P.my, z = r / P.my;
      const size_t i0 = g << 2;
      float w[3][4] = {};
      stress_div4(P, n, aligned, x0, y, z, i0, a1x, a1y, a1z, a4x, a4y, a4z, w);
#pragma unroll
      for (int comp = 0; comp < 3; ++comp) {
        float4 d = make_float4(w[comp][0], w[comp][1], w[comp][2], w[comp][3]);
        if (set) {
          const float4 d1 = *reinterpret_cast<const float4*>(R.ndiv + comp * nc + i0);
          d = make_float4(d1.x + d.x, d1.y + d.y, d1.z + d.z, d1.w + d.w);
        }
        *reinterpret_cast<float4*>(D + comp * nc + i0) = d;
      }
    }
    return;
  }
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nc; i += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % P.mx), r = (int)(i / P.mx);
    const int y = r % P.my, z = r / P.my;
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      float d = stress_div(P, n, comp, x, y, z, (int)i, a1x, a1y, a1z, a4x, a4y, a4z);
      if (set) d = R.ndiv[comp * nc + i] + d;
      D[comp * nc + i] = d;
    }
  }
}

static void launch_div(const Batch& B, int set, cudaStream_t s) {
  const int tb = 256;
  const long work = (B.mx & 3) == 0 ? (long)B.nc / 4 : (long)B.nc;
  long blocks = (work + tb - 1) / tb;
  const long cap = (148L * 16 + B.nrep - 1) / B.nrep;
  if (blocks > cap) blocks = cap < 1 ? 1 : cap;
  FSL_GO(k_div, dim3((unsigned)blocks, B.nrep), tb, 0, s, B, set);
}

void launch_noise(const Batch& B, cudaStream_t s, int scheme, int part) {
  const bool div = B.prec != PREC_F64 && scheme <= 1;
  if (part != 0) {
    // the second stress sample's divergence, after the first's
    if (div && scheme == 0) launch_div(B, 1, s);
    return;
  }
  if (B.prec == PREC_F64) return launch_noise64(B, s);
  const int tb = 256;
  uint64_t nb = (B.max_noise_n + 3) / 4;
  unsigned bx = blocks_for((long)nb, tb);
  unsigned cap = (unsigned)((148 * 16 + B.nrep - 1) / B.nrep);
  if (bx > cap) bx = cap < 1 ? 1 : cap;
  FSL_GO(k_noise, dim3(bx, B.nrep), tb, 0, s, B);
  if (div) launch_div(B, 0, s);
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
template <bool ONE>
__global__ void k_zero_cells(FSL_KARGS) {
  FSL_REP_AT(blockIdx.y);
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < P.mN; c += gridDim.x * blockDim.x) {
    R.cnt[c] = 0;
    R.fill[c] = 0;
    if (P.np == 0) R.start[c] = 0;  // no scan follows for an empty instance
  }
  if (P.np == 0 && blockIdx.x == 0 && threadIdx.x == 0) R.start[P.mN] = 0;
}

// one particle of each phase of the build (the kernels below, and the
// cooperative single-launch build)
__device__ __forceinline__ void cell_count_one(const Rep& R, int i, int which) {
  const Params& P = R.P;
  const double* q = which ? R.qp : R.q;
  double x = q[i], y = q[P.np + i], z = q[2 * P.np + i];
  // a coordinate this large or non-finite means the run has blown up
  const double lim = 1e15;
  if (!(fabs(x) < lim && fabs(y) < lim && fabs(z) < lim)) set_err(R.err, 2);
  const double wx = minimage(x, P.invlx, P.lx), wy = minimage(y, P.invly, P.ly),
               wz = minimage(z, P.invlz, P.lz);
  int c = cellidx(wx, P.invdnx, P.mnx) + cellidx(wy, P.invdny, P.mny) * P.mnx +
          cellidx(wz, P.invdnz, P.mnz) * P.mnx * P.mny;
  R.cell_of[i] = c;
  if (R.qw) {  // the pair loop works on wrapped positions
    R.qw[i] = wx;
    R.qw[P.np + i] = wy;
    R.qw[2 * P.np + i] = wz;
  }
  atomicAdd(&R.cnt[c], 1);
}

template <bool ONE>
__global__ void k_cell_count(FSL_KARGS, int which) {
  FSL_REP_FLAT(KIND_T1);
  int i = blk * blockDim.x + threadIdx.x;
  if (i >= P.np || !list_needed(R, which)) return;
  cell_count_one(R, i, which);
}

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ void block_scan(const int (&v)[kScanItems], int& incl_out, int& sum_out,
                                           int* warp_tot, int& total) {
  int sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) sum += v[k];
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
    if (lane == 31) warp_tot[32] = wi;
  }
  __syncthreads();
  incl_out = warp_tot[warp] + incl - sum;  // exclusive prefix of this thread
  sum_out = sum;
  total = warp_tot[32];
}

// Block-local exclusive scan of cnt into start, block totals into bsum.  The
// counts are cleared behind the read, ready for the next build.
template <bool ONE>
__global__ void __launch_bounds__(kScanThreads) k_scan_local(FSL_KARGS, int which) {
  FSL_REP_AT(blockIdx.y);
  if (!list_needed(R, which)) return;
  int* start = which && R.start1 ? R.start1 : R.start;
  __shared__ int warp_tot[33];
  const int n = P.mN;
  int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) v[k] = (base + k < n) ? R.cnt[base + k] : 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) R.cnt[base + k] = 0;
  int run, sum, total;
  block_scan(v, run, sum, warp_tot, total);
  if (threadIdx.x == 0) R.bsum[blockIdx.x] = total;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) start[base + k] = run;
    run += v[k];
  }
}

// Adds to every tile of start the sum of the block totals of the tiles
// before it (a block reduction of at most kScanTile totals), and writes the
// grand total to start[mN].
template <bool ONE>
__global__ void __launch_bounds__(kScanThreads) k_scan_add(FSL_KARGS, int which) {
  FSL_REP_AT(blockIdx.y);
  if (!list_needed(R, which)) return;
  int* start = which && R.start1 ? R.start1 : R.start;
  __shared__ int warp_sum[32];
  const int tile = blockIdx.x;
  int part = 0;
  for (int k = threadIdx.x; k < tile; k += blockDim.x) part += R.bsum[k];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = part;
  __syncthreads();
  int prefix = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) prefix += warp_sum[w];
  const int n = P.mN;
  const int base = tile * kScanTile + threadIdx.x * kScanItems;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) start[base + k] += prefix;
  if (threadIdx.x == 0 && tile == (n + kScanTile - 1) / kScanTile - 1) start[n] = prefix + R.bsum[tile];
}

// The slot checks below keep every write inside the cell's bucket even when
// the counts and starts disagree (a single-launch build whose grid barrier
// gave up leaves them so); such a write is skipped and flagged.
__device__ __forceinline__ void cell_scatter_one(const Rep& R, int i, int which) {
  const int* start = which && R.start1 ? R.start1 : R.start;
  int c = R.cell_of[i];
  const int k = start[c] + atomicAdd(&R.fill[c], 1);
  if (k >= start[c] && k < start[c + 1]) R.tmp[k] = i;
  else set_err(R.err, 4);
}

template <bool ONE>
__global__ void k_cell_scatter(FSL_KARGS, int which) {
  FSL_REP_FLAT(KIND_T1);
  int i = blk * blockDim.x + threadIdx.x;
  if (i >= P.np || !list_needed(R, which)) return;
  cell_scatter_one(R, i, which);
}

// Rank of particle i among the particles of its cell = number of smaller
// indices in the (unordered) bucket; gives the ascending order.
__device__ __forceinline__ void cell_rank_one(const Rep& R, int i, int which) {
  const Params& P = R.P;
  const bool second = which && R.start1;
  const int* start = second ? R.start1 : R.start;
  int* sorted = second ? R.sorted1 : R.sorted;
  double* ws = second ? R.ws1 : R.ws;
  int c = R.cell_of[i];
  int s = start[c], e = start[c + 1];
  int rank = 0;
  for (int k = s; k < e; ++k) rank += R.tmp[k] < i;
  R.fill[c] = 0;  // the scatter's slot counters, cleared for the next build
  if (s + rank >= e) {  // counts and starts disagree (see cell_scatter_one)
    set_err(R.err, 4);
    return;
  }
  sorted[s + rank] = i;
  if (ws) {  // wrapped positions in cell order for the pair loop
    ws[s + rank] = R.qw[i];
    ws[P.np + s + rank] = R.qw[P.np + i];
    ws[2 * P.np + s + rank] = R.qw[2 * P.np + i];
  }
}

template <bool ONE>
__global__ void k_cell_rank(FSL_KARGS, int which) {
  FSL_REP_FLAT(KIND_T1);
  int i = blk * blockDim.x + threadIdx.x;
  if (i >= P.np || !list_needed(R, which)) return;
  cell_rank_one(R, i, which);
}

void launch_cells(const Batch& B, int which, cudaStream_t s, bool zero_first) {
  const int tb = kPartThreads;
  if (zero_first) {
    unsigned zb = blocks_for(B.mN, tb);
    if (zb > 1024) zb = 1024;
    FSL_GO(k_zero_cells, dim3(zb, B.nrep), tb, 0, s, B);
  }
  if (B.max_np == 0) return;
  const unsigned pb = part_blocks(B, KIND_T1);
  FSL_GO(k_cell_count, pb, tb, 0, s, B, which);
  const unsigned nblk = blocks_for(B.mN, kScanTile);
  FSL_GO(k_scan_local, dim3(nblk, B.nrep), kScanThreads, 0, s, B, which);
  FSL_GO(k_scan_add, dim3(nblk, B.nrep), kScanThreads, 0, s, B, which);
  FSL_GO(k_cell_scatter, pb, tb, 0, s, B, which);
  FSL_GO(k_cell_rank, pb, tb, 0, s, B, which);
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

// Pair (src/stokesLimitFunctions.cu:191-653 with the table of
// src/initForcesNonBonded.cu:21-66, or soft repulsion) and bonded
// (src/forceBondedGPU.cu:21-121) force on every particle.  Eight lanes per
// particle, particles taken in cell order.  The lanes concatenate the
// candidate lists of the 27 neighbour cells (an exclusive scan of the cell
// counts in shared memory) and take candidates sub, sub+8, ... of the whole
// list, so the work is split evenly whatever the cell occupancy; candidates
// are read from the positions wrapped and stored in cell order by the cell
// list build.  The partial forces are summed in a fixed butterfly order.
template <bool ONE>
__global__ void __launch_bounds__(kPartThreads, 4) k_forces(FSL_KARGS, int which) {
  FSL_REP_FLAT(KIND_T8);
  __shared__ int s_pre[kPartThreads / 8][28];
  __shared__ int s_st[kPartThreads / 8][27];
  const int sub = threadIdx.x & 7, grp = threadIdx.x >> 3;
  const int ig = (int)((blk * (size_t)blockDim.x + threadIdx.x) >> 3);  // rank in cell order
  if ((ig & ~3) >= P.np) return;  // uniform per warp (4 particles per warp)
  const bool active = ig < P.np;  // inactive lanes still join the shuffles
  const int np = P.np;
  if (P.verlet || P.nolist) return;  // k_forces_vl
  // first-order scheme: forces at q^{n+1/2} only with extraMobility
  // (src/boundaryParticlesFunctionStokesLimitFirstOrder.cu:170-180)
  if (which == 1 && P.scheme == 1 && !P.has_extra) return;
  const CellList cl = cell_list(R, which);
  const int i = active ? cl.sorted[ig] : 0;
  const double* __restrict__ q = which ? R.qp : R.q;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  if (P.bonded && active) {
    const double rx = q[i], ry = q[np + i], rz = q[2 * np + i];
    int nb = R.bpp_cnt[i], off = R.bpp_off[i];
    for (int j = sub; j < nb; j += 8) {
      int idx = R.bpp_idx[off + j];
      bond_force(rx, ry, rz, q[idx], q[np + idx], q[2 * np + idx], R.bpp_k[off + j],
                 R.bpp_r0[off + j], fx, fy, fz);
    }
    nb = R.bfp_cnt[i];
    off = R.bfp_off[i];
    for (int j = sub; j < nb; j += 8) {
      const double* p = R.bfp_xyz + 3 * (off + j);
      bond_force(rx, ry, rz, p[0], p[1], p[2], R.bfp_k[off + j], R.bfp_r0[off + j], fx, fy, fz);
    }
  }
  if (P.nonbonded && P.pair != 0) {
    const double* __restrict__ ws = cl.ws;  // wrapped, cell order
    const double wx = active ? ws[ig] : 0.0, wy = active ? ws[np + ig] : 0.0,
                 wz = active ? ws[2 * np + ig] : 0.0;
    // the cell of the wrapped position, the arithmetic of k_cell_count (no
    // dependence on the load of i)
    const int c = cellidx(wx, P.invdnx, P.mnx) + cellidx(wy, P.invdny, P.mny) * P.mnx +
                  cellidx(wz, P.invdnz, P.mnz) * P.mnx * P.mny;
    const int cxy = c % (P.mnx * P.mny);
    const int cz = c / (P.mnx * P.mny), cy = cxy / P.mnx, cx = cxy - cy * P.mnx;
    // this lane's cells nn = sub + 8 m, in z-major order
    int st[4], cnt[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int nn = sub + 8 * m;
      st[m] = 0;
      cnt[m] = 0;
      if (active && nn < 27) {
        int ox = cx + nn % 3 - 1, oy = cy + (nn / 3) % 3 - 1, oz = cz + nn / 9 - 1;
        ox += ox < 0 ? P.mnx : (ox >= P.mnx ? -P.mnx : 0);
        oy += oy < 0 ? P.mny : (oy >= P.mny ? -P.mny : 0);
        oz += oz < 0 ? P.mnz : (oz >= P.mnz ? -P.mnz : 0);
        const int cc = ox + oy * P.mnx + oz * P.mnx * P.mny;
        st[m] = cl.start[cc];
        cnt[m] = cl.start[cc + 1] - st[m];
      }
    }
    // exclusive scan of the 27 counts in cell order, within the 8 lanes
    int carry = 0;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      int incl = cnt[m];
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o, 8);
        if (sub >= o) incl += y;
      }
      if (sub + 8 * m < 27) {
        s_pre[grp][sub + 8 * m] = carry + incl - cnt[m];
        s_st[grp][sub + 8 * m] = st[m];
      }
      carry += __shfl_sync(0xffffffffu, incl, 7, 8);
    }
    const int K = carry;
    if (sub == 0) s_pre[grp][27] = K;
    __syncwarp();
    const double c1 = 2.0 * P.soft_eps / P.cutoff, c2 = 1.0 / P.cutoff;
    int cp = 0;
    for (int kk = sub; kk < K; kk += 8) {
      while (s_pre[grp][cp + 1] <= kk) ++cp;
      const int jj = s_st[grp][cp] + (kk - s_pre[grp][cp]);
      const double rxij = minimage_near(wx - ws[jj], P.invlx, P.lx);
      const double ryij = minimage_near(wy - ws[np + jj], P.invly, P.ly);
      const double rzij = minimage_near(wz - ws[2 * np + jj], P.invlz, P.lz);
      // no fused multiply-add: r^2 selects the table entry bit-exactly
      const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(rxij, rxij), __dmul_rn(ryij, ryij)),
                                  __dmul_rn(rzij, rzij));
      double f;
      if (P.pair == 1) {
        f = (double)tex_linear(R.ljtab, kLjTableSize, (float)(r2 * P.invcut2));
      } else {
        if (jj == ig || r2 >= P.cutoff2 || r2 == 0.0) continue;
        // (2 eps / rc) (1 - r / rc) / r = c1 (1/r - 1/rc)
        f = c1 * (rsqrt(r2) - c2);
      }
      fx += f * rxij;
      fy += f * ryij;
      fz += f * rzij;
    }
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
  }
  if (sub != 0 || !active) return;
  if (!isfinite(fx) || !isfinite(fy) || !isfinite(fz)) set_err(R.err, 2);
  R.F[i] = fx;
  R.F[np + i] = fy;
  R.F[2 * np + i] = fz;
}

// ------------------------------------------------------------ Verlet list ---
// Soft repulsion has an explicit cutoff, so its pair forces can come from a
// list of the pairs within rc + skin at reference positions qref: every pair
// within rc at positions that moved at most skin / 2 from qref is on it.
// The list is rebuilt from a cell list of the current positions (the cells
// are at least rc wide, so the pairs within rc + skin <= 2 rc lie within two
// cells) when the update kernels have flagged a particle that moved further,
// after positions were set from the host, and at the first evaluation.
// Neighbours are stored in the cell order of the scan (deterministic).
__device__ void vl_build_one(const Rep& R, int i, int which) {
  const Params& P = R.P;
  const int np = P.np;
  const CellList cl = cell_list(R, which);
  const double* __restrict__ q = which ? R.qp : R.q;
  const double xi = q[i], yi = q[np + i], zi = q[2 * np + i];
  const double wx = minimage(xi, P.invlx, P.lx), wy = minimage(yi, P.invly, P.ly),
               wz = minimage(zi, P.invlz, P.lz);
  const int cx = cellidx(wx, P.invdnx, P.mnx), cy = cellidx(wy, P.invdny, P.mny),
            cz = cellidx(wz, P.invdnz, P.mnz);
  // per direction the cells within two of the particle's, each once
  const int nx = min(P.mnx, 5), ny = min(P.mny, 5), nz = min(P.mnz, 5);
  const int bx = P.mnx <= 5 ? 0 : cx - 2, by = P.mny <= 5 ? 0 : cy - 2, bz = P.mnz <= 5 ? 0 : cz - 2;
  int n = 0;
  bool over = false;
  for (int oz = 0; oz < nz; ++oz) {
    const int z = wrap_add(bz, oz, P.mnz);
    for (int oy = 0; oy < ny; ++oy) {
      const int y = wrap_add(by, oy, P.mny);
      for (int ox = 0; ox < nx; ++ox) {
        const int c = wrap_add(bx, ox, P.mnx) + P.mnx * (y + P.mny * z);
        for (int e = cl.start[c]; e < cl.start[c + 1]; ++e) {
          const int j = cl.sorted[e];
          if (j == i) continue;
          const double rx = minimage(xi - q[j], P.invlx, P.lx);
          const double ry = minimage(yi - q[np + j], P.invly, P.ly);
          const double rz = minimage(zi - q[2 * np + j], P.invlz, P.lz);
          if (rx * rx + ry * ry + rz * rz >= P.vl_cut2) continue;
          if (n < kVlCap) R.vl_idx[(size_t)n * np + i] = j;
          else over = true;
          ++n;
        }
      }
    }
  }
  R.vl_cnt[i] = min(n, kVlCap);
  R.qref[i] = xi;
  R.qref[np + i] = yi;
  R.qref[2 * np + i] = zi;
  if (over) R.vl_flag[2] = 3;  // cell mode from now on
}

template <bool ONE>
__global__ void k_vl_build(FSL_KARGS, int which) {
  FSL_REP_FLAT(KIND_T1);
  const int i = blk * blockDim.x + threadIdx.x;
  if (i >= P.np || !P.verlet || !list_needed(R, which) || R.vl_flag[2] == 3) return;
  vl_build_one(R, i, which);
}

// Positions replaced from the host: the Verlet list is rebuilt at the next
// evaluation at q only if a particle now lies more than skin / 2 from its
// reference position (a host loop that feeds back the positions it read
// keeps its list).
__global__ void k_moved_check(const __grid_constant__ Rep R) {
  const Params& P = R.P;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.np; i += gridDim.x * blockDim.x) {
    const double dx = R.q[i] - R.qref[i], dy = R.q[P.np + i] - R.qref[P.np + i],
                 dz = R.q[2 * P.np + i] - R.qref[2 * P.np + i];
    if (dx * dx + dy * dy + dz * dz > P.vl_half2) R.vl_flag[0] = *R.t + 1;
  }
}

void launch_moved_check(const Rep& r, cudaStream_t s) {
  if (!r.P.verlet || r.P.np == 0) return;
  const unsigned b = (unsigned)std::min<long>(148L * 4, ((long)r.P.np + 255) / 256);
  k_moved_check<<<b, 256, 0, s>>>(r);
}

// ----------------------------------------------- single-launch list build ---
// The cell list (and the Verlet list) of one instance in one cooperative
// launch: the phases of the kernels above separated by grid barriers, so a
// force evaluation that needs no rebuild costs one near-empty launch instead
// of six.  The barrier spins with a bound (spin_limit waits of 64 ns); if it
// gives up (the blocks are co-resident by the cooperative launch, so it
// should not) the block sets FSL_ERRBIT_GRID in the instance's error word and
// stops, and every other block stops at its next barrier.  The lists are then
// incomplete but every access stays in bounds (the slot checks of the scatter
// and rank phases); the build is skipped while the bit is set, and
// fsl_clear_errors clears the counters and the barrier and requests a fresh
// build.
// 1024 threads per block: one block per SM at the kernel's 48 registers, so
// that the common launch, which returns at once because no rebuild is due,
// schedules 148 blocks instead of 740 (about 3 µs a step less)
constexpr int kCoopThreads = 1024;
constexpr long kCoopSpinLimit = 20000000L;  // about a second

__device__ __forceinline__ bool grid_aborted(const Rep& R) {
  return (reinterpret_cast<volatile int*>(R.err)[ERR_BITS] & 4) != 0;
}

// false: this block must stop (its own wait gave up, or another block's did)
__device__ bool grid_barrier(const Rep& R, long spin_limit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = R.bar + 1;
    const unsigned g = *gen;
    __threadfence();
    int ok = 1;
    if (atomicAdd(R.bar, 1u) == gridDim.x - 1) {
      R.bar[0] = 0u;
      __threadfence();
      atomicAdd(R.bar + 1, 1u);
    } else {
      long spins = 0;
      while (*gen == g) {
        if (++spins > spin_limit) {
          set_err(R.err, 4);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_ok = ok && !grid_aborted(R);
  }
  __syncthreads();
  return s_ok != 0;
}

__global__ void __launch_bounds__(kCoopThreads) k_lists_coop(const __grid_constant__ Rep R, int which,
                                                             long spin_limit) {
  const Params& P = R.P;
  if (!R.active || P.np == 0 || !list_needed(R, which) || grid_aborted(R)) return;
  const int np = P.np, nb = gridDim.x;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = nb * blockDim.x;
  for (int i = tid; i < np; i += nth) cell_count_one(R, i, which);
  if (!grid_barrier(R, spin_limit)) return;
  // exclusive scan of the counts: block b takes a contiguous chunk, the
  // block totals go through bsum, the counts are cleared behind the read
  int* start = which && R.start1 ? R.start1 : R.start;
  __shared__ int wsum[kCoopThreads / 32];
  __shared__ int s_off;
  const int n = P.mN, chunk = (n + nb - 1) / nb;
  const int c0 = min(n, blockIdx.x * chunk), c1 = min(n, c0 + chunk);
  const int per = (c1 - c0 + blockDim.x - 1) / blockDim.x;
  const int t0 = min(c1, c0 + (int)threadIdx.x * per), t1 = min(c1, t0 + per);
  int sum = 0;
  for (int c = t0; c < t1; ++c) sum += R.cnt[c];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  int woff = 0, btot = 0;
  for (int w = 0; w < kCoopThreads / 32; ++w) {
    if (w < warp) woff += wsum[w];
    btot += wsum[w];
  }
  if (threadIdx.x == 0) R.bsum[blockIdx.x] = btot;
  if (!grid_barrier(R, spin_limit)) return;
  if (threadIdx.x == 0) {
    int off = 0;
    for (int b = 0; b < (int)blockIdx.x; ++b) off += R.bsum[b];
    s_off = off;
    if (blockIdx.x == nb - 1) start[n] = off + btot;
  }
  __syncthreads();
  int run = s_off + woff + incl - sum;
  for (int c = t0; c < t1; ++c) {
    const int v = R.cnt[c];
    start[c] = run;
    R.cnt[c] = 0;
    run += v;
  }
  if (!grid_barrier(R, spin_limit)) return;
  for (int i = tid; i < np; i += nth) cell_scatter_one(R, i, which);
  if (!grid_barrier(R, spin_limit)) return;
  for (int i = tid; i < np; i += nth) cell_rank_one(R, i, which);
  if (!P.verlet) return;
  if (!grid_barrier(R, spin_limit)) return;
  if (R.vl_flag[2] == 3) return;  // cell mode: no pair list
  for (int i = tid; i < np; i += nth) vl_build_one(R, i, which);
}

// ------------------------------------------- block-per-instance list build ---
// The lists of every instance of a batch of small instances in one launch:
// block r runs the phases of the separate kernels above for instance r, with
// block barriers between them (count, exclusive scan tile by tile with a
// running carry, scatter, rank, Verlet list).  Each phase leaves the words
// the separate kernels leave (the rank phase orders every cell by particle
// index whatever order the scatter's atomics took), so the lists are the
// same, and a force evaluation of a batch costs one launch instead of six.
// Taken for batches whose instances have at most kBlockListsMaxNp particles
// and kBlockListsMaxCells cells (a block of 1024 threads per instance keeps
// each phase to a few passes); larger instances keep the separate kernels,
// whose grids spread an instance over many blocks.
constexpr int kBlockListsMaxNp = 8192;
constexpr int kBlockListsMaxCells = 1 << 18;

template <bool ONE>
__global__ void __launch_bounds__(kScanThreads) k_lists_block(FSL_KARGS, int which) {
  FSL_REP_AT(blockIdx.x);
  if (!list_needed(R, which)) return;
  const int np = P.np, n = P.mN;
  for (int i = threadIdx.x; i < np; i += blockDim.x) cell_count_one(R, i, which);
  __syncthreads();
  int* start = which && R.start1 ? R.start1 : R.start;
  __shared__ int warp_tot[33];
  int carry = 0;
  for (int tile = 0; tile < n; tile += kScanTile) {
    const int base = tile + threadIdx.x * kScanItems;
    int v[kScanItems];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) v[k] = (base + k < n) ? R.cnt[base + k] : 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
      if (base + k < n) R.cnt[base + k] = 0;
    int run, sum, total;
    block_scan(v, run, sum, warp_tot, total);
    run += carry;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      if (base + k < n) start[base + k] = run;
      run += v[k];
    }
    carry += total;
    __syncthreads();  // every thread has read warp_tot before the next tile writes it
  }
  if (threadIdx.x == 0) start[n] = carry;
  __syncthreads();
  for (int i = threadIdx.x; i < np; i += blockDim.x) cell_scatter_one(R, i, which);
  __syncthreads();
  for (int i = threadIdx.x; i < np; i += blockDim.x) cell_rank_one(R, i, which);
  if (!P.verlet) return;
  __syncthreads();
  if (R.vl_flag[2] == 3) return;  // cell mode: no pair list
  for (int i = threadIdx.x; i < np; i += blockDim.x) vl_build_one(R, i, which);
}

int block_lists_env() {
  static const int v = [] {
    const char* e = getenv("FLUAMSL_BLOCK_LISTS");
    return !e || !*e ? -1 : e[0] == '0' ? 0 : 1;
  }();
  return v;
}

bool block_lists_eligible(const Batch& B) {
  return !B.one && B.max_np > 0 && B.max_np <= kBlockListsMaxNp && B.mN <= kBlockListsMaxCells;
}

bool block_lists(const Batch& B) {
  const int env = block_lists_env();
  if (!block_lists_eligible(B) || env == 0) return false;
  return env == 1 || B.lists_pick != 0;
}

static void lists_separate(const Batch& B, int which, cudaStream_t s);

void lists_autotune(const Batch& B, cudaStream_t s, float us[2]) {
  us[0] = us[1] = 0.f;
  if (!block_lists_eligible(B)) return;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    cudaGetLastError();
    return;
  }
  // three rounds over the two builds in turn, three builds each after one
  // untimed, the fastest round kept
  float best[2] = {1e30f, 1e30f};
  for (int round = 0; round < 3; ++round)
    for (int k = 0; k < 2; ++k) {
      auto build = [&] {
        if (k) FSL_GO(k_lists_block, dim3(B.nrep), kScanThreads, 0, s, B, 0);
        else lists_separate(B, 0, s);
      };
      build();
      cudaEventRecord(e0, s);
      for (int r = 0; r < 3; ++r) build();
      cudaEventRecord(e1, s);
      float ms = 0.f;
      if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) ms = 1e9f;
      best[k] = std::min(best[k], ms * 1000.f / 3.f);
    }
  us[0] = best[0];
  us[1] = best[1];
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGetLastError();
}

// The pair (Verlet list, or the 27 cells of the current cell list in cell
// mode) and bonded force on particle i by its quad: lane a takes list
// entries and bonds a, a + 4, ...; the partial forces are summed in a fixed
// butterfly order, every lane of the quad gets the sum.  Every lane of the
// warp calls this (shuffles); lanes with on == false contribute nothing.
__device__ __forceinline__ void quad_force_vl(const Params& P, const Rep& R, int i, int a, int which,
                                              bool on, bool cell_mode, double& fx, double& fy,
                                              double& fz) {
  const int np = P.np;
  const double* __restrict__ q = which ? R.qp : R.q;
  const double rx = q[i], ry = q[np + i], rz = q[2 * np + i];
  fx = 0.0;
  fy = 0.0;
  fz = 0.0;
  if (P.bonded && on) {
    int nb = R.bpp_cnt[i], off = R.bpp_off[i];
    for (int j = a; j < nb; j += 4) {
      const int idx = R.bpp_idx[off + j];
      bond_force(rx, ry, rz, q[idx], q[np + idx], q[2 * np + idx], R.bpp_k[off + j], R.bpp_r0[off + j],
                 fx, fy, fz);
    }
    nb = R.bfp_cnt[i];
    off = R.bfp_off[i];
    for (int j = a; j < nb; j += 4) {
      const double* p = R.bfp_xyz + 3 * (off + j);
      bond_force(rx, ry, rz, p[0], p[1], p[2], R.bfp_k[off + j], R.bfp_r0[off + j], fx, fy, fz);
    }
  }
  if (P.verlet && on && cell_mode) {
    // the 27 neighbour cells of the current cell list, lanes taking cells
    // a, a + 4, ...
    const double c1 = 2.0 * P.soft_eps / P.cutoff, c2 = 1.0 / P.cutoff;
    const CellList cl = cell_list(R, which);
    const int cx = cellidx(minimage(rx, P.invlx, P.lx), P.invdnx, P.mnx),
              cy = cellidx(minimage(ry, P.invly, P.ly), P.invdny, P.mny),
              cz = cellidx(minimage(rz, P.invlz, P.lz), P.invdnz, P.mnz);
    for (int nn = a; nn < 27; nn += 4) {
      const int c = wrap_add(cx, nn % 3 - 1, P.mnx) +
                    P.mnx * (wrap_add(cy, (nn / 3) % 3 - 1, P.mny) + P.mny * wrap_add(cz, nn / 9 - 1, P.mnz));
      for (int e2 = cl.start[c]; e2 < cl.start[c + 1]; ++e2) {
        const int j = cl.sorted[e2];
        const double rxij = minimage(rx - q[j], P.invlx, P.lx);
        const double ryij = minimage(ry - q[np + j], P.invly, P.ly);
        const double rzij = minimage(rz - q[2 * np + j], P.invlz, P.lz);
        const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(rxij, rxij), __dmul_rn(ryij, ryij)),
                                    __dmul_rn(rzij, rzij));
        if (j == i || r2 >= P.cutoff2 || r2 == 0.0) continue;
        const double f = c1 * (rsqrt(r2) - c2);
        fx += f * rxij;
        fy += f * ryij;
        fz += f * rzij;
      }
    }
  } else if (P.verlet && on) {
    const double c1 = 2.0 * P.soft_eps / P.cutoff, c2 = 1.0 / P.cutoff;
    const int n = R.vl_cnt[i];
    for (int k = a; k < n; k += 4) {
      const int j = R.vl_idx[(size_t)k * np + i];
      const double rxij = minimage(rx - q[j], P.invlx, P.lx);
      const double ryij = minimage(ry - q[np + j], P.invly, P.ly);
      const double rzij = minimage(rz - q[2 * np + j], P.invlz, P.lz);
      const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(rxij, rxij), __dmul_rn(ryij, ryij)),
                                  __dmul_rn(rzij, rzij));
      if (r2 >= P.cutoff2 || r2 == 0.0) continue;
      const double f = c1 * (rsqrt(r2) - c2);
      fx += f * rxij;
      fy += f * ryij;
      fz += f * rzij;
    }
  }
#pragma unroll
  for (int o = 1; o < 4; o <<= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
  }
}

// Whether the instance is in cell mode, read by every thread of the block
// before block 0 clears the rebuild request (the lists were rebuilt by the
// launch before); all threads of the block call this.
__device__ __forceinline__ bool vl_state(const Rep& R, int blk) {
  const bool cell_mode = R.P.verlet && R.vl_flag[2] == 3;
  __syncthreads();  // every thread has read the word before it is cleared
  if (blk == 0 && threadIdx.x == 0 && R.vl_flag && !cell_mode) R.vl_flag[2] = 0;  // rebuilt by now
  return cell_mode;
}

// Pair forces from the Verlet list (soft repulsion with the cutoff test and
// arithmetic of k_forces, on the minimum image of the unwrapped positions as
// the reference takes it) plus the bonded forces; one quad per particle
// (quad_force_vl).  Also the force kernel of instances without pair forces
// (bonds only).  Where a spread follows at the same positions, k_spread
// computes these forces itself instead.
template <bool ONE>
__global__ void k_forces_vl(FSL_KARGS, int which) {
  FSL_REP_FLAT(KIND_T4);
  long e;
  int a, qb;
  const int np = P.np;
  if (!(P.verlet || P.nolist)) return;
  const bool cell_mode = vl_state(R, blk);
  if (!quad_of(blk, np, e, a, qb)) return;
  // first-order scheme: forces at q^{n+1/2} only with extraMobility
  // (src/boundaryParticlesFunctionStokesLimitFirstOrder.cu:170-180)
  if (which == 1 && P.scheme == 1 && !P.has_extra) return;
  const bool on = e < np;
  const int i = on ? (int)e : 0;
  double fx, fy, fz;
  quad_force_vl(P, R, i, a, which, on, cell_mode, fx, fy, fz);
  if (!on || a != 0) return;
  if (!isfinite(fx) || !isfinite(fy) || !isfinite(fz)) set_err(R.err, 2);
  R.F[i] = fx;
  R.F[np + i] = fy;
  R.F[2 * np + i] = fz;
}

void launch_forces(const Batch& B, int which, cudaStream_t s, bool vl) {
  if (B.max_np == 0) return;
  if (B.has_cl) FSL_GO(k_forces, part_blocks(B, KIND_T8), kPartThreads, 0, s, B, which);
  if (B.has_vl && vl) FSL_GO(k_forces_vl, part_blocks(B, KIND_T4), kPartThreads, 0, s, B, which);
}

// Blocks of the cooperative build: all co-resident, computed once per device
// (host threads on different devices each read their own entry).
static unsigned coop_blocks() {
  constexpr int kMaxDev = 64;
  static std::atomic<unsigned> cache[kMaxDev];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < kMaxDev) {
    const unsigned c = cache[dev].load(std::memory_order_relaxed);
    if (c) return c;
  }
  int per_sm = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lists_coop, kCoopThreads, 0);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long b = (long)per_sm * sms;
  const unsigned blocks = (unsigned)std::max(1L, std::min(b, (long)kCoopMaxBlocks));
  if (dev >= 0 && dev < kMaxDev) cache[dev].store(blocks, std::memory_order_relaxed);
  return blocks;
}

// The wait bound of the cooperative build's grid barriers; the variable
// FLUAMSL_COOP_SPIN_LIMIT overrides it (the failure-path test sets 0, so that
// every wait gives up at once).
static long coop_spin_limit() {
  const char* e = getenv("FLUAMSL_COOP_SPIN_LIMIT");
  return e && *e ? atol(e) : kCoopSpinLimit;
}

cudaError_t launch_pair_lists(const Batch& B, int which, cudaStream_t s) {
  if (B.one && B.one->bar && B.max_np > 0) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(coop_blocks());
    cfg.blockDim = dim3(kCoopThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_lists_coop, *B.one, which, coop_spin_limit());
  }
  if (block_lists(B)) {
    FSL_GO(k_lists_block, dim3(B.nrep), kScanThreads, 0, s, B, which);
    return cudaPeekAtLastError();
  }
  lists_separate(B, which, s);
  return cudaPeekAtLastError();
}

static void lists_separate(const Batch& B, int which, cudaStream_t s) {
  launch_cells(B, which, s, false);
  if (B.max_np > 0 && B.has_vl) FSL_GO(k_vl_build, part_blocks(B, KIND_T1), kPartThreads, 0, s, B, which);
}

// After an error: the cell-list counters and the grid barrier of the
// single-launch build back to zero (a build that gave up leaves them
// partial).
__global__ void k_reset_lists(const __grid_constant__ Rep R) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < R.P.mN; c += gridDim.x * blockDim.x) {
    R.cnt[c] = 0;
    R.fill[c] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && R.bar) {
    R.bar[0] = 0u;
    R.bar[1] = 0u;
  }
}

void launch_reset_lists(const Rep& r, cudaStream_t s) {
  if (!r.cnt) return;
  unsigned b = blocks_for(r.P.mN, 256);
  if (b > 1024) b = 1024;
  k_reset_lists<<<std::max(b, 1u), 256, 0, s>>>(r);
}

// ------------------------------------------------------------ quad layout ---
// Spreading and interpolation take four lanes per particle (eight particles
// per warp).  Lane a = lane & 3 of a quad computes node a of the six stencil
// families (the cell-centre and face node families of each dimension),
// keeps its own x nodes and takes all y and z nodes of the quad by
// shuffles; it then handles x node a of every stencil, the KN^2 (y, z)
// nodes of each component (a = 3 idles for the 3-point kernel).  A warp
// instruction touches eight particles' x-runs of four consecutive values.
template <int KN>
struct QuadStencil {
  int jx[2], jy[2][KN], jz[2][KN];  // family 0: cell centres, 1: faces
  float wx[2], wy[2][KN], wz[2][KN];
};

// The nodes and weights that lane a of a quad computes itself: node a of
// family f (0: cell centres, 1: faces) in dimension d (zeros for a >= KN).
struct QuadLane {
  int j[2][3];
  float w[2][3];
};

template <int KN>
__device__ __forceinline__ void quad_lane(const Params& P, const double posc[3], const double posw[3], int a,
                                          QuadLane& L) {
#pragma unroll
  for (int f = 0; f < 2; ++f)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      L.j[f][d] = 0;
      L.w[f][d] = 0.0f;
      if (a < KN) stencil_node(P, d, f == 1 ? d : (d + 1) % 3, posc[d], posw[d], a, L.j[f][d], L.w[f][d]);
    }
}

// The quad's stencil from its lanes' own nodes: x stays with its lane, y and
// z go to every lane of the quad (first lane qb).
template <int KN>
__device__ __forceinline__ void quad_share(const QuadLane& L, int qb, QuadStencil<KN>& S) {
#pragma unroll
  for (int f = 0; f < 2; ++f) {
    S.jx[f] = L.j[f][0];
    S.wx[f] = L.w[f][0];
#pragma unroll
    for (int k = 0; k < KN; ++k) {
      S.jy[f][k] = __shfl_sync(0xffffffffu, L.j[f][1], qb + k);
      S.wy[f][k] = __shfl_sync(0xffffffffu, L.w[f][1], qb + k);
      S.jz[f][k] = __shfl_sync(0xffffffffu, L.j[f][2], qb + k);
      S.wz[f][k] = __shfl_sync(0xffffffffu, L.w[f][2], qb + k);
    }
  }
}

template <int KN>
__device__ __forceinline__ void quad_stencil(const Params& P, const double posc[3],
                                             const double posw[3], int a, int qb,
                                             QuadStencil<KN>& S) {
  QuadLane L;
  quad_lane<KN>(P, posc, posw, a, L);
  quad_share<KN>(L, qb, S);
}

// The stencil cache of the midpoint scheme: lane slot (particle i, lane a)
// = 4 i + a of 4 np slots per plane, three 16-byte planes
// A = (j00 j01 j02 j10), B = (j11 j12 w00 w01), C = (w02 w10 w11 w12).
__device__ __forceinline__ void lane_store(uint4* stc, size_t np4, size_t slot, const QuadLane& L) {
  stc[slot] = make_uint4((unsigned)L.j[0][0], (unsigned)L.j[0][1], (unsigned)L.j[0][2], (unsigned)L.j[1][0]);
  stc[np4 + slot] =
      make_uint4((unsigned)L.j[1][1], (unsigned)L.j[1][2], __float_as_uint(L.w[0][0]), __float_as_uint(L.w[0][1]));
  stc[2 * np4 + slot] = make_uint4(__float_as_uint(L.w[0][2]), __float_as_uint(L.w[1][0]),
                                   __float_as_uint(L.w[1][1]), __float_as_uint(L.w[1][2]));
}

__device__ __forceinline__ void lane_load(const uint4* __restrict__ stc, size_t np4, size_t slot, QuadLane& L) {
  const uint4 A = __ldg(stc + slot), B = __ldg(stc + np4 + slot), C = __ldg(stc + 2 * np4 + slot);
  L.j[0][0] = (int)A.x;
  L.j[0][1] = (int)A.y;
  L.j[0][2] = (int)A.z;
  L.j[1][0] = (int)A.w;
  L.j[1][1] = (int)B.x;
  L.j[1][2] = (int)B.y;
  L.w[0][0] = __uint_as_float(B.z);
  L.w[0][1] = __uint_as_float(B.w);
  L.w[0][2] = __uint_as_float(C.x);
  L.w[1][0] = __uint_as_float(C.y);
  L.w[1][1] = __uint_as_float(C.z);
  L.w[1][2] = __uint_as_float(C.w);
}

// One spread of one particle by its quad: every lane adds w * value of its
// nodes in 64-bit fixed point (in the float-atomic form: w * value as an
// FP32 atomic).  Replaces the slot writes of
// kernelSpreadParticlesForceStokesLimit and kernelSpreadParticlesDrift + the
// gather of addSpreadedForcesStokesLimit (src/stokesLimitFunctions.cu:
// 659-1681, 1705-2255); the 1/dV of the gather is applied when the field is
// read back.  No shuffles: lanes may skip it.
template <int KN>
__device__ __forceinline__ void quad_spread(const Params& P, const QuadStencil<KN>& S, int a,
                                            const double val[3],
                                            unsigned long long* __restrict__ grid, bool& sat) {
  if (a >= KN) return;
  const bool fatom = P.prec == PREC_FLOAT;
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
    const double vc = val[comp];
    if (vc == 0.0) continue;  // every product is zero: nothing to add
    const int x = S.jx[comp == 0];
    const float wx = S.wx[comp == 0];
    const double vs = vc * kFixedScale;
    unsigned long long* gc = grid + (size_t)comp * P.nc;
#pragma unroll
    for (int b = 0; b < KN; ++b) {
      const int y = S.jy[comp == 1][b];
      const float wy = S.wy[comp == 1][b];
#pragma unroll
      for (int c = 0; c < KN; ++c) {
        const int at = x + P.mx * (y + P.my * S.jz[comp == 2][c]);  // < nc <= 2^30
        const float w = wx * (wy * S.wz[comp == 2][c]);
        if (fatom) {
          // float-atomic form: the first 3 nc floats of the spread buffer
          const float fv = (float)((double)w * vc);
          if (fv != 0.0f) atomicAdd(reinterpret_cast<float*>(grid) + (size_t)comp * P.nc + at, fv);
          continue;
        }
        const double v = (double)w * vs;
        sat |= !(fabs(v) < kFixedMax);
        const long long iv = sat ? 0ll : __double2ll_rn(v);
        if (iv != 0) atomicAdd(gc + at, (unsigned long long)iv);
      }
    }
  }
}

// J v of one particle by its quad: each lane sums w v over its nodes per
// component, then the quad adds its four partial sums (xor 1, then xor 2);
// every lane of the quad gets the three sums
// (src/stokesLimitFunctions.cu:2616-2642).
template <int KN>
__device__ __forceinline__ void quad_interp(const Params& P, const QuadStencil<KN>& S, int a,
                                            const float* __restrict__ v, float u[3]) {
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
    const float* vc = v + (size_t)comp * P.nc;
    const int x = S.jx[comp == 0];
    const float wx = S.wx[comp == 0];
    float val[KN * KN];
#pragma unroll
    for (int b = 0; b < KN; ++b)
#pragma unroll
      for (int c = 0; c < KN; ++c)
        val[b * KN + c] = a < KN ? __ldg(vc + (x + P.mx * (S.jy[comp == 1][b] + P.my * S.jz[comp == 2][c]))) : 0.0f;
    float s = 0.0f;
#pragma unroll
    for (int b = 0; b < KN; ++b)
#pragma unroll
      for (int c = 0; c < KN; ++c) s += (wx * (S.wy[comp == 1][b] * S.wz[comp == 2][c])) * val[b * KN + c];
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    u[comp] = s;
  }
}


// The RFD drift of particle i by its quad: (kT/delta) sign W_p spread from
// q + sign (delta/2) W_p for both signs through add(stencil, values).  In
// reference mode the drift's nodes come from the displaced position and its
// weights from q, as the reference does; where both displaced positions pick
// the same nodes the two fixed-point spreads are exact negatives of each
// other (same weights, opposite values, symmetric rounding), so they are
// skipped without changing the result.  Every lane of the warp calls this.
__device__ __forceinline__ void rfd_inputs(const Params& P, const Rep& R, int i, double W[3],
                                           double pos[3]) {
  const int np = P.np;
  const size_t wbase = (size_t)6 * P.nc;
  W[0] = (double)R.noise[wbase + i];
  W[1] = (double)R.noise[wbase + np + i];
  W[2] = (double)R.noise[wbase + 2 * np + i];
  pos[0] = R.q[i];
  pos[1] = R.q[np + i];
  pos[2] = R.q[2 * np + i];
}

// W: the particle's RFD noise, pos: q^n (rfd_inputs)
template <int KN, class Add>
__device__ __forceinline__ void rfd_drift_at(const Params& P, const double W[3], const double pos[3],
                                             int a, int qb, bool on, Add&& add) {
  double pp[3], pm[3], vp[3], vm[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    pp[d] = pos[d] + 0.5 * kRfdDelta * W[d];
    pm[d] = pos[d] - 0.5 * kRfdDelta * W[d];
    vp[d] = (P.kT / kRfdDelta) * W[d];
    vm[d] = (P.kT / kRfdDelta) * -1 * W[d];
  }
  QuadStencil<KN> S;
  if (P.rfd != 1) {
    // lane a checks the node families a and a + 4 of the six (bit f 3 + d
    // of chg: family f of dimension d picks another first node)
    int chg = 0;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int fd = a + 4 * r;
      if (fd < 6) {
        const int f = fd / 3, d = fd - 3 * f;
        const double x = d == 0 ? pp[0] : (d == 1 ? pp[1] : pp[2]);
        const double y = d == 0 ? pm[0] : (d == 1 ? pm[1] : pm[2]);
        if (stencil_base(P, d, f, x) != stencil_base(P, d, f, y)) chg |= 1 << fd;
      }
    }
    chg |= __shfl_xor_sync(0xffffffffu, chg, 1);
    chg |= __shfl_xor_sync(0xffffffffu, chg, 2);
    const bool same = chg == 0;
    if (!__all_sync(0xffffffffu, same || !on)) {
      // component c reads the face family of dimension c and the centre
      // families of the other two; a component none of whose families
      // changed has the same nodes and weights in both spreads, which then
      // cancel exactly: its values are left at zero (quad_spread skips them)
      constexpr int fam[3] = {(1 << 3) | (1 << 1) | (1 << 2), (1 << 4) | (1 << 0) | (1 << 2),
                              (1 << 5) | (1 << 0) | (1 << 1)};
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (!(chg & fam[c])) vp[c] = vm[c] = 0.0;
      quad_stencil<KN>(P, pp, pos, a, qb, S);
      if (on && !same) add(S, vp);
      quad_stencil<KN>(P, pm, pos, a, qb, S);
      if (on && !same) add(S, vm);
    }
  } else {
    quad_stencil<KN>(P, pp, pp, a, qb, S);
    if (on) add(S, vp);
    quad_stencil<KN>(P, pm, pm, a, qb, S);
    if (on) add(S, vm);
  }
}

template <int KN, class Add>
__device__ __forceinline__ void rfd_drift(const Params& P, const Rep& R, int i, int a, int qb,
                                          bool on, Add&& add) {
  double W[3], pos[3];
  rfd_inputs(P, R, i, W, pos);
  rfd_drift_at<KN>(P, W, pos, a, qb, on, add);
}

// ------------------------------------------------- warp-aggregated spread ---
// The fixed-point spread of a warp's eight particles gathered in a shared
// box before it reaches the L2: consecutive particles (a chain's beads, or
// cell-ordered particles) share most stencil nodes, and the L2 takes 64-bit
// atomic adds at a limited rate.  Per component the warp finds the box of
// kBox^3 nodes that holds the stencils of its live particles (relative to
// the first particle's nodes, periodic); each product goes into the box as
// two 32-bit shared atomics (low word, then high word plus the carry of the
// low one: exact integer arithmetic mod 2^64, so every node's sum is the
// same integer whatever the order); the box is then flushed with one 64-bit
// global atomic per non-zero node and left cleared.  A warp whose particles do not fit in the box, and
// grids with fewer than kBox cells along an axis, take the per-particle
// atomics of quad_spread.  Same products (w = wx (wy wz) times the
// fixed-point value), same integer sums: bitwise equal to quad_spread.
constexpr int kBox = 8;
constexpr int kBoxNodes = kBox * kBox * kBox;

// d wrapped into [-m/2, m/2)
__device__ __forceinline__ int rel_wrap(int d, int m) {
  if (2 * d >= m) d -= m;
  else if (2 * d < -m) d += m;
  return d;
}

template <int KN>
__device__ __forceinline__ void warp_spread(const Params& P, const QuadStencil<KN>& S, int a,
                                            const double val[3], bool on,
                                            unsigned long long* __restrict__ grid, bool& sat,
                                            unsigned* __restrict__ blo, unsigned* __restrict__ bhi) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const bool small = P.mx < kBox || P.my < kBox || P.mz < kBox;
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
    // first node of the quad per dimension: x of lane 0 of the quad, y and z
    // shared by the quad's lanes
    const int x0 = __shfl_sync(full, S.jx[comp == 0], lane & ~3);
    const int y0 = S.jy[comp == 1][0], z0 = S.jz[comp == 2][0];
    const int X0 = __shfl_sync(full, x0, 0), Y0 = __shfl_sync(full, y0, 0),
              Z0 = __shfl_sync(full, z0, 0);
    const int dx = rel_wrap(x0 - X0, P.mx), dy = rel_wrap(y0 - Y0, P.my), dz = rel_wrap(z0 - Z0, P.mz);
    constexpr int kBig = 1 << 28;
    const int lx = __reduce_min_sync(full, on ? dx : kBig), hx = __reduce_max_sync(full, on ? dx : -kBig);
    const int ly = __reduce_min_sync(full, on ? dy : kBig), hy = __reduce_max_sync(full, on ? dy : -kBig);
    const int lz = __reduce_min_sync(full, on ? dz : kBig), hz = __reduce_max_sync(full, on ? dz : -kBig);
    const bool fits = !small && hx - lx + KN <= kBox && hy - ly + KN <= kBox && hz - lz + KN <= kBox;
    const double vs = val[comp] * kFixedScale;
    if (!fits) {  // warp-uniform
      if (on && a < KN) {
        unsigned long long* gc = grid + (size_t)comp * P.nc;
        const int x = S.jx[comp == 0];
        const float wx = S.wx[comp == 0];
#pragma unroll
        for (int b = 0; b < KN; ++b)
#pragma unroll
          for (int c = 0; c < KN; ++c) {
            const int at = x + P.mx * (S.jy[comp == 1][b] + P.my * S.jz[comp == 2][c]);
            const float w = wx * (S.wy[comp == 1][b] * S.wz[comp == 2][c]);
            const double v = (double)w * vs;
            sat |= !(fabs(v) < kFixedMax);
            const long long iv = sat ? 0ll : __double2ll_rn(v);
            if (iv != 0) atomicAdd(gc + at, (unsigned long long)iv);
          }
      }
      continue;
    }
    if (on && a < KN) {
      const float wx = S.wx[comp == 0];
      const int bx = dx - lx + a;
#pragma unroll
      for (int b = 0; b < KN; ++b)
#pragma unroll
        for (int c = 0; c < KN; ++c) {
          const float w = wx * (S.wy[comp == 1][b] * S.wz[comp == 2][c]);
          const double v = (double)w * vs;
          sat |= !(fabs(v) < kFixedMax);
          const long long iv = sat ? 0ll : __double2ll_rn(v);
          // unconditional (a zero adds nothing): straight-line code lets
          // the low-word adds of the stencil issue back to back
          const int n = ((dz - lz + c) * kBox + (dy - ly + b)) * kBox + bx;
          const unsigned lo = (unsigned)(unsigned long long)iv;
          const unsigned hi = (unsigned)((unsigned long long)iv >> 32);
          const unsigned old = atomicAdd(blo + n, lo);
          atomicAdd(bhi + n, hi + (old + lo < old ? 1u : 0u));
        }
    }
    __syncwarp();
    // the box's first node, in [0, m); m >= kBox, so one wrap per axis
    int bx0 = X0 + lx, by0 = Y0 + ly, bz0 = Z0 + lz;
    bx0 += bx0 < 0 ? P.mx : (bx0 >= P.mx ? -P.mx : 0);
    by0 += by0 < 0 ? P.my : (by0 >= P.my ? -P.my : 0);
    bz0 += bz0 < 0 ? P.mz : (bz0 >= P.mz ? -P.mz : 0);
    unsigned long long* gc = grid + (size_t)comp * P.nc;
#pragma unroll 4
    for (int n = lane; n < kBoxNodes; n += 32) {
      const unsigned lo = blo[n], hi = bhi[n];
      if ((lo | hi) == 0u) continue;
      blo[n] = 0u;
      bhi[n] = 0u;
      int x = bx0 + (n & (kBox - 1)), y = by0 + ((n / kBox) & (kBox - 1)), z = bz0 + n / (kBox * kBox);
      x -= x >= P.mx ? P.mx : 0;
      y -= y >= P.my ? P.my : 0;
      z -= z >= P.mz ? P.mz : 0;
      atomicAdd(gc + x + P.mx * (y + P.my * z), ((unsigned long long)hi << 32) | lo);
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------- spreading ---
// One quad per particle (in cell order when ordered).  drift = 0: F at q;
// drift = 1: F at q^{n+1/2}, then the particle's RFD drift (kT/delta) sign
// W_p from q + sign (delta/2) W_p for both signs; drift = 2: F at q and the
// drift.  In reference mode the drift's nodes come from the displaced
// position and its weights from q, as the reference does.
template <bool ONE, int KN>
__global__ void __launch_bounds__(kPartThreads, 4) k_spread(FSL_KARGS, int drift, int ordered, int box, int forces, int cache) {
  FSL_REP_FLAT(KIND_T4);
  // the warp's aggregation box (low and high words), kept cleared
  __shared__ unsigned s_box[kPartThreads / 32][2][kBoxNodes];
  long e;
  int a, qb;
  const int np = P.np;
  // forces: the Verlet-list and bonded forces at the spread's positions are
  // computed here (k_forces_vl's arithmetic) and stored, instead of read
  const bool own_forces = forces && (P.verlet || P.nolist);
  const bool cell_mode = own_forces ? vl_state(R, blk) : false;
  if (!quad_of(blk, np, e, a, qb)) return;
  const bool on = e < np;  // lanes past the end join the shuffles only
  // cell order on the cell-list path (a list the step has just built)
  const bool by_cell = ordered && !P.verlet && !P.nolist;
  const int i = on ? (by_cell ? cell_list(R, drift == 1).sorted[e] : (int)e) : 0;
  bool sat = false;
  QuadStencil<KN> S;
  {
    const double* qf = drift == 1 ? R.qp : R.q;
    double pos[3] = {qf[i], qf[np + i], qf[2 * np + i]};
    double val[3];
    if (own_forces) {
      quad_force_vl(P, R, i, a, drift == 1 ? 1 : 0, on, cell_mode, val[0], val[1], val[2]);
      if (on && a == 0) {
        if (!isfinite(val[0]) || !isfinite(val[1]) || !isfinite(val[2])) set_err(R.err, 2);
        R.F[i] = val[0];
        R.F[np + i] = val[1];
        R.F[2 * (size_t)np + i] = val[2];
      }
    } else {
      val[0] = R.F[i];
      val[1] = R.F[np + i];
      val[2] = R.F[2 * (size_t)np + i];
    }
    {
      QuadLane L;
      quad_lane<KN>(P, pos, pos, a, L);
      // the interpolation at the same positions takes these nodes back
      if (cache && on && R.stc) lane_store(R.stc, (size_t)4 * np, (size_t)4 * i + a, L);
      quad_share<KN>(L, qb, S);
    }
    if (P.prec == PREC_FIXED && box) {
      unsigned* blo = s_box[threadIdx.x >> 5][0];
      unsigned* bhi = s_box[threadIdx.x >> 5][1];
      for (int n = threadIdx.x & 31; n < kBoxNodes; n += 32) {
        blo[n] = 0u;
        bhi[n] = 0u;
      }
      __syncwarp();
      warp_spread<KN>(P, S, a, val, on, R.grid, sat, blo, bhi);
    } else if (on) {
      quad_spread<KN>(P, S, a, val, R.grid, sat);
    }
  }
  if (drift) {
    // the RFD drift of the same particle, by the same quad
    rfd_drift<KN>(P, R, i, a, qb, on, [&](const QuadStencil<KN>& T, const double val[3]) {
      quad_spread<KN>(P, T, a, val, R.grid, sat);
    });
  }
  if (sat) set_err(R.err, 1);
}

// FLUAMSL_SPREAD_BOX=0 spreads every product with its own global atomic (the
// same sums, for comparison)
static int spread_box() {
  static const int on = [] {
    const char* e = getenv("FLUAMSL_SPREAD_BOX");
    return (e && e[0] == '0') ? 0 : 1;
  }();
  return on;
}

void launch_spread(const Batch& B, int drift, int ordered, cudaStream_t s, bool forces, bool cache) {
  if (B.max_np == 0) return;
  if (B.prec == PREC_F64) return launch_spread64(B, drift, s);
  const unsigned g = part_blocks(B, KIND_T4);
  const int f = forces ? 1 : 0, c = cache ? 1 : 0;
  if (B.kernel == 4)
    FSL_GO_T(k_spread, 4, g, kPartThreads, 0, s, B, drift, ordered, spread_box(), f, c);
  else
    FSL_GO_T(k_spread, 3, g, kPartThreads, 0, s, B, drift, ordered, spread_box(), f, c);
}

// ------------------------------------------------ tiled spread + W build ---
// The fixed-point form's spread and W build in one pass, without the spread
// field in HBM.  A block owns a tile of kTileX x kTileY x kTileZ cells: it
// takes from the cell lists every particle whose stencils can reach the
// tile, adds the fixed-point products of the stencil nodes inside the tile
// with shared-memory 64-bit atomics (the same integers the global spread
// adds, so every node's sum is the same integer), then builds W = f +
// c div(Sigma) of its cells with the arithmetic of k_wbuild4 (k_wbuild when
// mx is not a multiple of 4) and stores it with coalesced 16-byte writes.
// Replaces the slot writes and gathers of the reference's spreading
// (src/stokesLimitFunctions.cu:659-1681, 1705-2255) and
// kernelConstructWstokesLimit(_2) (:2281-2378, 3922-4069).

constexpr int kTileX = 32, kTileY = 8, kTileZ = 8;
constexpr int kTileCells = kTileX * kTileY * kTileZ;
constexpr int kTileThreads = 256;
constexpr int kTileMaxRuns = 1024;
constexpr int kTileChunk = 1024;  // candidates filtered per round

// Neighbour cells [a, b] (up to two intervals after the periodic wrap, no
// cell twice) holding every particle whose stencil nodes can reach the cells
// [x0, x1) of a grid of m cells: a stencil node lies within H cells of the
// particle's grid coordinate, and one neighbour cell more on each side
// absorbs the rounding of the cell assignment.
struct NbRange {
  int n, a[2], b[2];
  __host__ __device__ int cells() const { return (b[0] - a[0] + 1) + (n > 1 ? b[1] - a[1] + 1 : 0); }
  __host__ __device__ int at(int k) const { return k <= b[0] - a[0] ? a[0] + k : a[1] + k - (b[0] - a[0] + 1); }
};

__host__ __device__ inline int floor_div(long p, long q) {
  return (int)(p >= 0 ? p / q : -((-p + q - 1) / q));
}

__host__ __device__ inline NbRange nb_range(int x0, int x1, int m, int mn, int H) {
  const int lo = floor_div((long)(x0 - H) * mn, m) - 1;
  const int hi = floor_div((long)(x1 + H) * mn, m) + 1;
  NbRange r;
  r.n = 1;
  r.a[1] = r.b[1] = 0;
  if (hi - lo + 1 >= mn) {
    r.a[0] = 0;
    r.b[0] = mn - 1;
  } else if (lo < 0) {
    r.n = 2;
    r.a[0] = lo + mn;
    r.b[0] = mn - 1;
    r.a[1] = 0;
    r.b[1] = hi;
  } else if (hi >= mn) {
    r.n = 2;
    r.a[0] = lo;
    r.b[0] = mn - 1;
    r.a[1] = 0;
    r.b[1] = hi - mn;
  } else {
    r.a[0] = lo;
    r.b[0] = hi;
  }
  return r;
}

__host__ __device__ constexpr int tile_halo(int kn) { return kn / 2 + 2; }

size_t tile_smem_bytes() {
  return sizeof(unsigned long long) * 3 * kTileCells + sizeof(int) * (2 * kTileMaxRuns + 1 + kTileChunk);
}

// The runs of the block's candidates: for every (y, z) neighbour cell pair
// and x interval, the particles start[c(a, y, z)] .. start[c(b, y, z) + 1]
// of the cell-ordered list; run_pre gets the exclusive prefix of the run
// lengths (run_pre[nruns] = all candidates).  All threads call this.
__device__ void tile_runs(const int* __restrict__ start, const NbRange& ix, const NbRange& iy,
                          const NbRange& iz, int mnx, int mny, int* run_st, int* run_pre, int nruns) {
  const int ny = iy.cells();
  for (int r = threadIdx.x; r < nruns; r += blockDim.x) {
    const int xi = r % ix.n, pr = r / ix.n;
    const int y = iy.at(pr % ny), z = iz.at(pr / ny);
    const int row = mnx * (y + mny * z);
    const int s0 = start[ix.a[xi] + row];
    run_st[r] = s0;
    run_pre[r] = start[ix.b[xi] + row + 1] - s0;
  }
  __syncthreads();
  // exclusive scan: four entries per thread, then the threads' sums
  __shared__ int wsum[kTileThreads / 32];
  const int base = threadIdx.x * 4;
  int v[4], sum = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = base + k < nruns ? run_pre[base + k] : 0;
    sum += v[k];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  int off = 0;
  for (int w = 0; w < warp; ++w) off += wsum[w];
  int run = off + incl - sum;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (base + k < nruns) run_pre[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == blockDim.x - 1) run_pre[nruns] = run;
  __syncthreads();
}

// The products of the nodes of one spread that fall in the tile, added to
// the tile's accumulators (shared memory).  No shuffles.
template <int KN>
__device__ __forceinline__ void tile_spread(const Params& P, const QuadStencil<KN>& S, int a,
                                            const double val[3], unsigned long long* acc, int x0,
                                            int y0, int z0, bool& sat) {
  if (a >= KN) return;
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
    const int lx = S.jx[comp == 0] - x0;
    if ((unsigned)lx >= (unsigned)kTileX) continue;
    const float wx = S.wx[comp == 0];
    const double vs = val[comp] * kFixedScale;
    unsigned long long* ac = acc + comp * kTileCells + lx;
#pragma unroll
    for (int b = 0; b < KN; ++b) {
      const int ly = S.jy[comp == 1][b] - y0;
      if ((unsigned)ly >= (unsigned)kTileY) continue;
      const float wy = S.wy[comp == 1][b];
#pragma unroll
      for (int c = 0; c < KN; ++c) {
        const int lz = S.jz[comp == 2][c] - z0;
        if ((unsigned)lz >= (unsigned)kTileZ) continue;
        const float w = wx * (wy * S.wz[comp == 2][c]);
        const double v = (double)w * vs;
        sat |= !(fabs(v) < kFixedMax);
        const long long iv = sat ? 0ll : __double2ll_rn(v);
        if (iv != 0) atomicAdd(ac + (lz * kTileY + ly) * kTileX, (unsigned long long)iv);
      }
    }
  }
}

// drift: as k_spread (0: F at q; 1: F at q^{n+1/2} and the RFD drift at q^n;
// 2: F and the drift at q^n); the forces come from the list of their
// positions, the drift from the list at q^n.  nsets, nfac: the stress
// samples and factor of k_wbuild.
template <bool ONE, int KN>
__global__ void __launch_bounds__(kTileThreads) k_spread_w(FSL_KARGS, int drift, int nsets,
                                                            double nfac, int tiles_x, int tiles_y) {
  FSL_REP_AT(blockIdx.y);
  extern __shared__ unsigned long long tsm[];
  unsigned long long* acc = tsm;  // [3][kTileZ][kTileY][kTileX]
  int* run_st = reinterpret_cast<int*>(acc + 3 * kTileCells);
  int* run_pre = run_st + kTileMaxRuns;
  int* acc_list = run_pre + kTileMaxRuns + 1;  // [kTileChunk] accepted particles
  __shared__ int n_acc_s;
  int* n_acc = &n_acc_s;
  const int bt = blockIdx.x;
  const int x0 = (bt % tiles_x) * kTileX, y0 = ((bt / tiles_x) % tiles_y) * kTileY,
            z0 = (bt / (tiles_x * tiles_y)) * kTileZ;
  for (int k = threadIdx.x; k < 3 * kTileCells; k += blockDim.x) acc[k] = 0ull;
  bool sat = false;
  const int np = P.np;
  if (np > 0) {
    constexpr int H = tile_halo(KN);
    const NbRange ix = nb_range(x0, min(x0 + kTileX, P.mx), P.mx, P.mnx, H);
    const NbRange iy = nb_range(y0, min(y0 + kTileY, P.my), P.my, P.mny, H);
    const NbRange iz = nb_range(z0, min(z0 + kTileZ, P.mz), P.mz, P.mnz, H);
    const int nruns = ix.n * iy.cells() * iz.cells();  // <= kTileMaxRuns (checked on the host)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int a = lane & 3, qb = lane & ~3;
    auto add = [&](const QuadStencil<KN>& S, const double val[3]) {
      tile_spread<KN>(P, S, a, val, acc, x0, y0, z0, sat);
    };
    // a particle's stencil nodes lie within [u - 3, u + 1.5] (4-point) or
    // [u - 2.5, u + 1] (3-point) of its grid coordinate u; 0.05 more absorbs
    // the drift's displacement and rounding
    const double mlo = (KN == 4 ? 1.5 : 1.0) + 0.05, mhi = (KN == 4 ? 2.0 : 1.5) + 0.05;
    const int ex1 = min(x0 + kTileX, P.mx), ey1 = min(y0 + kTileY, P.my), ez1 = min(z0 + kTileZ, P.mz);
    auto near = [&](double w, double halfL, double invd, int lo, int hi, int m) {
      const double u = (w + halfL) * invd, a0 = lo - mlo, b0 = hi + mhi;
      return (u >= a0 && u < b0) || (u - m >= a0 && u - m < b0) || (u + m >= a0 && u + m < b0);
    };
    const int passes = drift == 1 ? 2 : 1;
    for (int pass = 0; pass < passes; ++pass) {
      const CellList cl = cell_list(R, drift == 1 && pass == 0 ? 1 : 0);
      __syncthreads();  // the runs and accepted list of the previous pass are read
      tile_runs(cl.start, ix, iy, iz, P.mnx, P.mny, run_st, run_pre, nruns);
      const int K = run_pre[nruns];
      for (int c0 = 0; c0 < K; c0 += kTileChunk) {
        // the candidates whose stencils can reach the tile, from their
        // wrapped positions in list order (the order of acceptance does not
        // matter: the fixed-point sums are exact)
        if (threadIdx.x == 0) *n_acc = 0;
        __syncthreads();
        const int c1 = min(K, c0 + kTileChunk);
        for (int k = c0 + threadIdx.x; k < c1; k += blockDim.x) {
          int lo = 0, hi = nruns;  // run_pre[lo] <= k < run_pre[hi]
          while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (run_pre[mid] <= k) lo = mid;
            else hi = mid;
          }
          const int e = run_st[lo] + (k - run_pre[lo]);
          if (near(cl.ws[e], 0.5 * P.lx, P.invdx, x0, ex1, P.mx) &&
              near(cl.ws[np + e], 0.5 * P.ly, P.invdy, y0, ey1, P.my) &&
              near(cl.ws[2 * np + e], 0.5 * P.lz, P.invdz, z0, ez1, P.mz))
            acc_list[atomicAdd(n_acc, 1)] = cl.sorted[e];
        }
        __syncthreads();
        const int na = *n_acc;
        for (int k0 = warp * 8; k0 < na; k0 += (kTileThreads / 32) * 8) {
          const int k = k0 + (lane >> 2);
          const bool on = k < na;
          const int i = on ? acc_list[k] : acc_list[0];
          if (pass == 0) {
            const double* qf = drift == 1 ? R.qp : R.q;
            double pos[3] = {qf[i], qf[np + i], qf[2 * np + i]};
            double val[3] = {R.F[i], R.F[np + i], R.F[2 * (size_t)np + i]};
            QuadStencil<KN> S;
            quad_stencil<KN>(P, pos, pos, a, qb, S);
            if (on) add(S, val);
          }
          if ((pass == 0 && drift == 2) || pass == 1) rfd_drift<KN>(P, R, i, a, qb, on, add);
        }
        __syncthreads();  // acc_list is read
      }
    }
  }
  __syncthreads();
  // W of the tile's cells
  const float scale = (float)(kFixedInv / P.dV);
  const float fac = (float)nfac;
  const size_t nc = (size_t)P.nc;
  const float* D = R.ndiv + (nsets > 1 ? 3 * nc : 0);
  const int ex = min(kTileX, P.mx - x0), ey = min(kTileY, P.my - y0), ez = min(kTileZ, P.mz - z0);
  if ((P.mx & 3) == 0) {
    constexpr int GX = kTileX / 4;
    for (int g = threadIdx.x; g < GX * kTileY * kTileZ; g += blockDim.x) {
      const int lx = 4 * (g % GX), ly = (g / GX) % kTileY, lz = g / (GX * kTileY);
      if (lx >= ex || ly >= ey || lz >= ez) continue;
      const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
      const size_t i0 = (size_t)x + (size_t)P.mx * ((size_t)y + (size_t)P.my * z);
      float w[3][4];
#pragma unroll
      for (int comp = 0; comp < 3; ++comp) {
        const float4 d4 = __ldg(reinterpret_cast<const float4*>(D + comp * nc + i0));
        const float d[4] = {d4.x, d4.y, d4.z, d4.w};
#pragma unroll
        for (int c = 0; c < 4; ++c)
          w[comp][c] = w_fixed((long long)acc[comp * kTileCells + (lz * kTileY + ly) * kTileX + lx + c], scale,
                               fac, d[c]);
      }
#pragma unroll
      for (int comp = 0; comp < 3; ++comp)
        *reinterpret_cast<float4*>(R.wbuf + comp * nc + i0) =
            make_float4(w[comp][0], w[comp][1], w[comp][2], w[comp][3]);
    }
  } else {
    for (int c = threadIdx.x; c < kTileCells; c += blockDim.x) {
      const int lx = c % kTileX, ly = (c / kTileX) % kTileY, lz = c / (kTileX * kTileY);
      if (lx >= ex || ly >= ey || lz >= ez) continue;
      const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
      const int i = x + P.mx * (y + P.my * z);
#pragma unroll
      for (int comp = 0; comp < 3; ++comp) {
        R.wbuf[comp * nc + i] = w_fixed((long long)acc[comp * kTileCells + c], scale, fac, __ldg(D + comp * nc + i));
      }
    }
  }
  if (sat) set_err(R.err, 1);
}

void tile_init() {
  const int sm = (int)tile_smem_bytes();
  cudaFuncSetAttribute(k_spread_w<true, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  cudaFuncSetAttribute(k_spread_w<true, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  cudaFuncSetAttribute(k_spread_w<false, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  cudaFuncSetAttribute(k_spread_w<false, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
}

bool pdl_enabled() {
  static const bool on = [] {
    const char* e = getenv("FLUAMSL_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}

bool tile_eligible(const Params& P) {
  if (P.prec != PREC_FIXED || P.scheme > 1) return false;  // 3-D Stokes schemes
  if (P.verlet || P.nolist) return false;  // needs both cell lists of every step
  // the drift's displacement (delta/2 |W| <= 0.003 for FP32 normals) must
  // stay well inside the candidates' spare 0.05 cells
  if (std::min(P.dx, std::min(P.dy, P.dz)) < 0.1) return false;
  // a block scans about (tile + 2 halo + 2 neighbour cells)^3: only worth it
  // while a neighbour cell spans at most four grid cells
  if (P.mx > 4 * P.mnx || P.my > 4 * P.mny || P.mz > 4 * P.mnz) return false;
  const int H = tile_halo(P.kernel);
  int runs = 1;
  const int m[3] = {P.mx, P.my, P.mz}, mn[3] = {P.mnx, P.mny, P.mnz}, t[3] = {kTileX, kTileY, kTileZ};
  for (int d = 0; d < 3; ++d) {
    int worst = 0;
    for (int x0 = 0; x0 < m[d]; x0 += t[d]) {
      const NbRange r = nb_range(x0, std::min(x0 + t[d], m[d]), m[d], mn[d], H);
      worst = std::max(worst, d == 0 ? r.n : r.cells());
    }
    runs *= worst;
  }
  return runs <= kTileMaxRuns;
}

void launch_spread_w(const Batch& B, int drift, int nsets, double nfac, cudaStream_t s) {
  const int tx = (B.mx + kTileX - 1) / kTileX, ty = (B.my + kTileY - 1) / kTileY,
            tz = (B.mz + kTileZ - 1) / kTileZ;
  const dim3 g((unsigned)(tx * ty * tz), (unsigned)B.nrep);
  const size_t sm = tile_smem_bytes();
  if (B.kernel == 4)
    FSL_GO_T(k_spread_w, 4, g, kTileThreads, sm, s, B, drift, nsets, nfac, tx, ty);
  else
    FSL_GO_T(k_spread_w, 3, g, kTileThreads, sm, s, B, drift, nsets, nfac, tx, ty);
}

// -------------------------------------------------------- interpolation ---
// stage 1: q^{n+1/2} = q^n + dt/2 J(q^n) v (+ extraMobility terms),
//          src/stokesLimitFunctions.cu:2646-2650
// stage 2: q^{n+1}   = q^n + dt J(q^{n+1/2}) v (+ extraMobility terms),
//          src/stokesLimitFunctions.cu:3676-3681
// One quad per particle; lanes 0, 1, 2 of the quad update x, y, z.
template <bool ONE, int KN>
__global__ void k_interp_update(FSL_KARGS, int stage, int cached) {
  FSL_REP_FLAT(KIND_T4);
  long e;
  int a, qb;
  const int np = P.np;
  if (!quad_of(blk, np, e, a, qb)) return;
  const bool on = e < np;
  const int i = on ? (int)e : 0;
  const double* qpos = stage == 1 ? R.q : R.qp;
  double* qout = stage == 1 ? R.qp : R.q;
  QuadStencil<KN> S;
  {
    // the nodes of the spread at the same positions, or computed here
    QuadLane L;
    if (cached && R.stc) {
      lane_load(R.stc, (size_t)4 * np, (size_t)4 * i + a, L);
    } else {
      double pos[3] = {qpos[i], qpos[np + i], qpos[2 * np + i]};
      quad_lane<KN>(P, pos, pos, a, L);
    }
    quad_share<KN>(L, qb, S);
  }
  float us[3];
  quad_interp<KN>(P, S, a, R.v, us);
  const int comp = a < 3 ? a : 0;
  const double u = (double)(comp == 0 ? us[0] : (comp == 1 ? us[1] : us[2]));
  size_t k = (size_t)comp * np + i;
  double h = stage == 1 ? 0.5 * P.dt : P.dt;
  double r = R.q[k] + h * u;
  if (P.has_extra) {
    size_t nb = (size_t)6 * P.nc + (size_t)(3 + comp) * np + i;
    double xi = (double)R.noise[nb];
    if (stage == 2) xi += (double)R.noise[nb + (size_t)3 * np];
    r += h * P.extra_mob * R.F[k] + P.fact2 * xi;
  }
  if (P.verlet) {
    // the Verlet list must be rebuilt before the next force evaluation
    // (at q^{n+1/2} in this step, or at q of the next) once a particle has
    // moved more than skin / 2 from its reference position
    const double d = a < 3 ? r - R.qref[k] : 0.0;
    double d2 = d * d;
    d2 += __shfl_xor_sync(0xffffffffu, d2, 1);
    d2 += __shfl_xor_sync(0xffffffffu, d2, 2);
    if (on && a == 0 && d2 > P.vl_half2) R.vl_flag[stage == 1 ? 1 : 0] = *R.t + stage;
  }
  if (!on || a >= 3) return;
  if (!isfinite(r)) set_err(R.err, 2);
  qout[k] = r;
}

template <bool ONE, int KN>
__global__ void k_interp(FSL_KARGS) {
  FSL_REP_FLAT(KIND_T4);
  long e;
  int a, qb;
  const int np = P.np;
  if (!quad_of(blk, np, e, a, qb)) return;
  const bool on = e < np;
  const int i = on ? (int)e : 0;
  double pos[3] = {R.q[i], R.q[np + i], R.q[2 * np + i]};
  QuadStencil<KN> S;
  quad_stencil<KN>(P, pos, pos, a, qb, S);
  float us[3];
  quad_interp<KN>(P, S, a, R.v, us);
  if (on && a < 3) R.u[(size_t)a * np + i] = (double)(a == 0 ? us[0] : (a == 1 ? us[1] : us[2]));
}

void launch_interp_update(const Batch& B, int stage, cudaStream_t s, bool cached) {
  if (B.max_np == 0) return;
  if (B.prec == PREC_F64) return launch_interp_update64(B, stage, s);
  const unsigned g = part_blocks(B, KIND_T4);
  const int c = cached ? 1 : 0;
  if (B.kernel == 4)
    FSL_GO_T(k_interp_update, 4, g, kPartThreads, 0, s, B, stage, c);
  else
    FSL_GO_T(k_interp_update, 3, g, kPartThreads, 0, s, B, stage, c);
}

void launch_interp(const Batch& B, cudaStream_t s) {
  if (B.max_np == 0) return;
  const unsigned g = part_blocks(B, KIND_T4);
  if (B.kernel == 4)
    FSL_GO_T(k_interp, 4, g, kPartThreads, 0, s, B);
  else
    FSL_GO_T(k_interp, 3, g, kPartThreads, 0, s, B);
}

template <bool ONE>
__global__ void k_step_counter(FSL_KARGS) {
  FSL_REP_AT(blockIdx.y);
  (void)P;
  if (threadIdx.x == 0) *R.t += 1;
}

void launch_step_counter(const Batch& B, cudaStream_t s) {
  FSL_GO(k_step_counter, dim3(1, B.nrep), 32, 0, s, B);
}

// ------------------------------------------------------------ observables ---
// FP64 sums over the particles (|q - q0|^2, q - q0, F) and the cells (v) of
// one instance.  Each block sums its share in a fixed order (grid-stride
// loops, butterfly within warps, warps in order) into its row of obs_part;
// the last block to finish, known by a ticket, adds the rows in block order
// and updates the accumulators, so the result does not depend on how the
// blocks were scheduled.
constexpr int kObsThreads = 256;

template <bool ONE>
__global__ void __launch_bounds__(kObsThreads) k_observe(FSL_KARGS) {
  FSL_REP_AT(blockIdx.y);
  if (!P.observe) return;
  __shared__ double red[kObsThreads / 32][kObsVals];
  __shared__ double tot[kObsVals];
  __shared__ int last;
  double acc[kObsVals];
#pragma unroll
  for (int k = 0; k < kObsVals; ++k) acc[k] = 0.0;
  const int np = P.np;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += stride) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double dd = R.q[(size_t)d * np + i] - R.q0[(size_t)d * np + i];
      acc[0] += dd * dd;
      acc[1 + d] += dd;
      acc[4 + d] += R.F[(size_t)d * np + i];
    }
  }
  const size_t nc = (size_t)P.nc;
  const bool f64 = P.prec == PREC_F64;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += stride)
      acc[7 + d] += f64 ? R.v64[d * nc + c] : (double)R.v[d * nc + c];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kObsVals; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if (lane == 0) red[warp][k] = acc[k];
  }
  __syncthreads();
  double* part = R.obs_part + (size_t)blockIdx.x * kObsVals;
  if (threadIdx.x < kObsVals) {
    double sum = 0.0;
    for (int w = 0; w < kObsThreads / 32; ++w) sum += red[w][threadIdx.x];
    part[threadIdx.x] = sum;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(R.obs_ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < kObsVals) {
    double sum = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b) sum += __ldcg(R.obs_part + (size_t)b * kObsVals + threadIdx.x);
    tot[threadIdx.x] = sum;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // steps, msd, msd_sum, displacement[3], force[3], momentum[3], momentum_sum[3]
    double* o = R.obs;
    const double inv_np = np > 0 ? 1.0 / np : 0.0;
    const double msd = tot[0] * inv_np;
    o[0] += 1.0;
    o[1] = msd;
    o[2] += msd;
    for (int d = 0; d < 3; ++d) {
      o[3 + d] = tot[1 + d] * inv_np;
      o[6 + d] = tot[4 + d];
      const double mom = tot[7 + d] * P.dV;
      o[9 + d] = mom;
      o[12 + d] += mom;
    }
    *R.obs_ticket = 0u;  // ready for the next launch
  }
}

void launch_observe(const Batch& B, cudaStream_t s) {
  long work = std::max<long>((long)B.max_np, (long)B.nc) / (kObsThreads * 16);
  const unsigned nb = (unsigned)std::min<long>(kObsMaxBlocks, std::max<long>(1, work));
  FSL_GO(k_observe, dim3(nb, B.nrep), kObsThreads, 0, s, B);
}

}  // namespace fsl
