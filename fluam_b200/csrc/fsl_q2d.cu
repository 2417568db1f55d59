// fsl_q2d.cu -- the quasi-2D family (FSL_SCHEME_QUASI2D, FSL_SCHEME_STOKES2D).
//
// The Gaussian-blob Stokes schemes of keywords quasi2D and stokesLimit2D
// (src/runSchemeQuasi2D.cu:20-260, src/quasi2DFunctions.cu) on a periodic
// mx x my grid, FP64 throughout as the reference.  Grid nodes sit at the
// cell corners x_k = k dx - lx/2; a particle's stencil is the (2w+1)^2 nodes
// around the node at or below it (w = kernelWidth).  One step: noise, the
// 2-D cell list and forces (only with computeNonBondedForces, as the
// reference), force and thermal-drift spreading with FP64 atomics into the
// real parts of the complex field, the optional shear forcing, a 2-D FFT,
// the Fourier-space mobility plus stochastic velocity per mode, the inverse
// FFT and the particle update (forward Euler or the predictor-corrector on
// the same velocity field).  The FFT passes are those of the FP64 form
// (fsl_fp64.cu); the cell list is the shared counting sort (one z layer).
#include "fsl_internal.cuh"

namespace fsl {

namespace {

unsigned blocks_for(long work, int tb) { return (unsigned)((work + tb - 1) / tb); }

constexpr double kPi = 3.1415926535897932385;
constexpr double kPiHalfInv = 0.56418958354775628695;  // 1 / sqrt(pi)

// src/deltaGPU.cu:114-117
__device__ __forceinline__ double gauss2d(double r2, double var) {
  return exp(-r2 / (2.0 * var)) / (2 * kPi * var);
}

// (k + o) mod m for any offset: the reference's (k + o + m) % m, which is the
// same whenever that argument is non-negative (a stencil wider than the grid
// in y would make it negative there)
__device__ __forceinline__ int node_wrap(int k, int o, int m) {
  int r = (k + o) % m;
  return r < 0 ? r + m : r;
}

// wrapped distance from coordinate r to node k (src/quasi2DFunctions.cu:262-270)
__device__ __forceinline__ double node_dist(double r, int k, double L, int m, double invL) {
  return minimage(r - (k * L / m) + L * 0.5, invL, L);
}

// ------------------------------------------------------------- forces ---
// One thread per particle: 2-D bonds (src/quasiNeutrallyBuoyantFunctions2D.cu:
// 201-260) and the pair force over the 9 neighbour cells of the 2-D cell
// list (src/quasi2DFunctions.cu:53-235), own cell first.
__device__ __forceinline__ void bond2d(double rx, double ry, double x, double y, double k,
                                       double r0, double& fx, double& fy) {
  if (r0 == 0) {
    fx += -k * (rx - x);
    fy += -k * (ry - y);
  } else {
    const double r = sqrt((x - rx) * (x - rx) + (y - ry) * (y - ry));
    if (r > 0) {
      fx += -k * (1 - r0 / r) * (rx - x);
      fy += -k * (1 - r0 / r) * (ry - y);
    }
  }
}

__device__ __forceinline__ float tex_linear2(const float* __restrict__ T, int N, float x) {
  double xb = (double)x * (double)N - 0.5;
  double fl = floor(xb);
  int i = (int)fl;
  float a = (float)(rint((xb - fl) * 256.0) * (1.0 / 256.0));
  int i0 = min(max(i, 0), N - 1);
  int i1 = min(max(i + 1, 0), N - 1);
  return __fadd_rn(__fmul_rn(1.0f - a, __ldg(T + i0)), __fmul_rn(a, __ldg(T + i1)));
}

template <bool ONE>
__global__ void k_q2_forces(FSL_KARGS) {
  FSL_REP_FLAT(KIND_T1);
  const int i = blk * blockDim.x + threadIdx.x;
  const int np = P.np;
  if (i >= np) return;
  const double* q = R.q;
  const double rx = q[i], ry = q[np + i];
  double fx = 0.0, fy = 0.0;
  // the reference computes no force at all without computeNonBondedForces
  // (the force kernel sits inside that test, src/runSchemeQuasi2D.cu:127-147)
  if (P.nonbonded && P.bonded) {
    const int nb = R.bpp_cnt[i], off = R.bpp_off[i];
    for (int j = 0; j < nb; ++j) {
      const int idx = R.bpp_idx[off + j];
      bond2d(rx, ry, q[idx], q[np + idx], R.bpp_k[off + j], R.bpp_r0[off + j], fx, fy);
    }
    const int nf = R.bfp_cnt[i], fo = R.bfp_off[i];
    for (int j = 0; j < nf; ++j) {
      const double* p = R.bfp_xyz + 3 * (fo + j);
      bond2d(rx, ry, p[0], p[1], R.bfp_k[fo + j], R.bfp_r0[fo + j], fx, fy);
    }
  }
  if (P.nonbonded && P.pair != 0) {
    const int c = R.cell_of[i];
    const int cx = c % P.mnx, cy = c / P.mnx;
    const double c1 = 2.0 * P.soft_eps / P.cutoff, c2 = 1.0 / P.cutoff;
    // own cell, -y, -x, +x, +y, (+x,+y), (+x,-y), (-x,+y), (-x,-y)
    const int ox[9] = {0, 0, -1, 1, 0, 1, 1, -1, -1};
    const int oy[9] = {0, -1, 0, 0, 1, 1, -1, 1, -1};
#pragma unroll 1
    for (int o = 0; o < 9; ++o) {
      const int nx = (cx + ox[o] + P.mnx) % P.mnx, ny = (cy + oy[o] + P.mny) % P.mny;
      const int cc = nx + ny * P.mnx;
      const int s = R.start[cc], e = R.start[cc + 1];
      for (int k = s; k < e; ++k) {
        const int j = R.sorted[k];
        const double rxij = minimage(rx - q[j], P.invlx, P.lx);
        const double ryij = minimage(ry - q[np + j], P.invly, P.ly);
        const double r2 = __dadd_rn(__dmul_rn(rxij, rxij), __dmul_rn(ryij, ryij));
        double f;
        if (P.pair == 1) {
          f = (double)tex_linear2(R.ljtab, kLjTableSize, (float)(r2 * P.invcut2));
        } else {
          if (j == i || r2 >= P.cutoff2 || r2 == 0.0) continue;
          f = c1 * (1.0 / sqrt(r2) - c2);
        }
        fx += f * rxij;
        fy += f * ryij;
      }
    }
  }
  if (!isfinite(fx) || !isfinite(fy)) set_err(R.err, 2);
  R.F[i] = fx;
  R.F[np + i] = fy;
  R.F[2 * (size_t)np + i] = 0.0;
}

// ----------------------------------------------------------- spreading ---
template <bool ONE>
__global__ void k_q2_zero(FSL_KARGS) {
  FSL_REP_AT(blockIdx.y);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 2 * (size_t)P.nc;
       i += (size_t)gridDim.x * blockDim.x)
    R.z64[i] = make_double2(0.0, 0.0);
}

// One thread per particle: g(r) F (with the forces) and the thermal drift
// -g(r) (kT / var) (r - x_node) (src/quasi2DFunctions.cu:243-281, 287-391)
// into the real parts of the two field components.
template <bool ONE>
__global__ void k_q2_spread(FSL_KARGS) {
  FSL_REP_FLAT(KIND_T1);
  const int i = blk * blockDim.x + threadIdx.x;
  const int np = P.np;
  if (i >= np) return;
  const int forces = P.nonbonded;
  if (!forces && !P.q2_rfd) return;
  const double rx = R.q[i], ry = R.q[np + i];
  const double fx = forces ? R.F[i] : 0.0, fy = forces ? R.F[np + i] : 0.0;
  const int mx = P.mx, my = P.my, w = P.q2_kw;
  const int kx = cellidx(minimage(rx, P.invlx, P.lx), P.invdx, mx);
  const int ky = cellidx(minimage(ry, P.invly, P.ly), P.invdy, my);
  double* zx = reinterpret_cast<double*>(R.z64);
  double* zy = reinterpret_cast<double*>(R.z64 + P.nc);
  for (int ix = -w; ix <= w; ++ix) {
    const int kxn = node_wrap(kx, ix, mx);
    const double dxr = node_dist(rx, kxn, P.lx, mx, P.invlx);
    for (int iy = -w; iy <= w; ++iy) {
      const int kyn = node_wrap(ky, iy, my);
      const double dyr = node_dist(ry, kyn, P.ly, my, P.invly);
      const double g = gauss2d(dxr * dxr + dyr * dyr, P.q2_var);
      const int c = kxn + kyn * mx;
      double ax = 0.0, ay = 0.0;
      if (forces) {
        ax += g * fx;
        ay += g * fy;
      }
      if (P.q2_rfd) {
        const double norm = g * P.kT / P.q2_var;
        ax += -norm * dxr;
        ay += -norm * dyr;
      }
      atomicAdd(zx + 2 * (size_t)c, ax);
      atomicAdd(zy + 2 * (size_t)c, ay);
    }
  }
}

// src/quasi2DFunctions.cu:3-12: vy += A sin(2 pi x / mx)
template <bool ONE>
__global__ void k_q2_shear(FSL_KARGS) {
  FSL_REP_AT(blockIdx.y);
  if (P.q2_shear == 0.0) return;
  const double pi2 = 2.0 * kPi;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.nc; i += gridDim.x * blockDim.x)
    R.z64[P.nc + i].x += P.q2_shear * sin(pi2 * ((i % P.mx) / (double)P.mx));
}

// ------------------------------------------------------ Fourier space ---
// Per mode: the mobility (RPY quasi-2D, src/quasi2DFunctions.cu:450-510;
// 2-D Stokes, :767-827; Saffman-screened, :966-1035) and the stochastic
// velocity with its Hermitian bookkeeping (:590-678, :829-904, :1037-1119).
template <bool ONE>
__global__ void k_q2_fourier(FSL_KARGS) {
  FSL_REP_AT(blockIdx.y);
  const int mx = P.mx, my = P.my, nc = P.nc, nModes = nc + mx + my;
  const double eta = P.eta, sigma = sqrt(P.q2_var), prefactor = P.q2_fact1;
  const bool rpy = P.scheme == 2;
  const double kc = P.q2_kc, lw = P.q2_lw;
  const double* Rn = R.noise64;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
    const double2 zx = R.z64[i], zy = R.z64[nc + i];
    // deterministic: signed wave numbers with the Nyquist rows folded
    double kx, ky;
    {
      int wy = i / mx, wx = i % mx;
      if (wx > mx / 2) wx -= mx;
      if (wy > my / 2) wy -= my;
      const bool xh = (mx % 2) == 0 && (wx == mx / 2);
      const bool yh = (my % 2) == 0 && (wy == my / 2);
      if (xh && wy < 0) wx *= -1;
      else if (yh && wx < 0) wy *= -1;
      kx = wx * 2 * kPi / P.lx;
      ky = wy * 2 * kPi / P.ly;
    }
    double oxr = 0, oxi = 0, oyr = 0, oyi = 0;
    if (i != 0) {
      if (rpy) {
        const double k_inv = 1.0 / sqrt(kx * kx + ky * ky);
        const double k3_inv = k_inv * k_inv * k_inv;
        const double k = 1.0 / k_inv, kn = sigma * k;
        const double f = 0.5 * (erfc(kn) * (0.5 + kn * kn) * exp(kn * kn) - kPiHalfInv * kn);
        const double g = 0.5 * erfc(kn) * exp(kn * kn);
        oxr = (k3_inv / eta) * (g * ky * (ky * zx.x - kx * zy.x) + f * kx * (kx * zx.x + ky * zy.x));
        oxi = (k3_inv / eta) * (g * ky * (ky * zx.y - kx * zy.y) + f * kx * (kx * zx.y + ky * zy.y));
        oyr = (k3_inv / eta) * (g * (-kx) * (ky * zx.x - kx * zy.x) + f * ky * (kx * zx.x + ky * zy.x));
        oyi = (k3_inv / eta) * (g * (-kx) * (ky * zx.y - kx * zy.y) + f * ky * (kx * zx.y + ky * zy.y));
      } else {
        const double L = -(kx * kx) - (ky * ky);
        double den;
        if (kc != 0.0) {
          const double kmod = sqrt(-L);
          const double corr = lw != 0.0 ? tanh(kmod * lw) : 1.0;
          den = eta * (kmod * (kmod + kc * corr));
        } else {
          den = -eta * L;
        }
        const double GWr = kx * zx.x + ky * zy.x, GWi = kx * zx.y + ky * zy.y;
        oxr = (zx.x + kx * GWr / L) / den;
        oxi = (zx.y + kx * GWi / L) / den;
        oyr = (zy.x + ky * GWr / L) / den;
        oyi = (zy.y + ky * GWi / L) / den;
      }
    }
    // stochastic: canonical |wave numbers|, the noise index shared with the
    // conjugate mode, and the flip of the conjugate's imaginary part
    int wy = i / mx, wx = i % mx, fx = wx, fy = wy, shift = 0;
    if (wx > mx / 2) {
      fx = wx - mx;
      wx = mx - wx;
    }
    if (wy > my / 2) {
      fy = wy - my;
      wy = my - wy;
    }
    const bool xHalf = (mx % 2) == 0 && (wx == mx / 2);
    const bool yHalf = (my % 2) == 0 && (wy == my / 2);
    if (xHalf && fy < 0) fx *= -1;
    else if (yHalf && fx < 0) fy *= -1;
    double mkx = wx * 2 * kPi / P.lx;
    const double mky = wy * 2 * kPi / P.ly;
    if (fx * fy < 0) {
      shift = nModes / 2;
      mkx *= -1.0;
    }
    const int index = wy * mx + wx + shift;
    const bool edge = (xHalf && wy == 0) || (yHalf && wx == 0) || (xHalf && yHalf);
    double Wxr = 0, Wxi = 0, Wyr = 0, Wyi = 0;
    if (rpy) {
      if (i != 0) {
        const double k = sqrt(mkx * mkx + mky * mky);
        const double k3half_inv = 1.0 / sqrt(k * k * k);
        const double kn = sigma * k;
        const double f_half = sqrt(0.5 * (erfc(kn) * (0.5 + kn * kn) * exp(kn * kn) - kPiHalfInv * kn));
        const double g_half = sqrt(0.5 * erfc(kn) * exp(kn * kn));
        const double a = g_half * mky, b = f_half * mkx, c = g_half * (-mkx), d = f_half * mky;
        if (edge) {
          Wxr = sqrt(2.0) * prefactor * k3half_inv * (a * Rn[index] + b * Rn[nModes + index]);
          Wyr = sqrt(2.0) * prefactor * k3half_inv * (c * Rn[index] + d * Rn[nModes + index]);
        } else {
          Wxr = prefactor * k3half_inv * (a * Rn[index] + b * Rn[nModes + index]);
          Wyr = prefactor * k3half_inv * (c * Rn[index] + d * Rn[nModes + index]);
          Wxi = prefactor * k3half_inv * (a * Rn[nModes * 2 + index] + b * Rn[nModes * 3 + index]);
          Wyi = prefactor * k3half_inv * (c * Rn[nModes * 2 + index] + d * Rn[nModes * 3 + index]);
        }
      }
    } else {
      const bool nyq = ((mx % 2) == 0 && (wx == mx / 2)) || ((my % 2) == 0 && (wy == my / 2)) || i == 0;
      if (!nyq) {
        double amp;
        if (kc != 0.0) {
          const double kmod2 = mkx * mkx + mky * mky, kmod = sqrt(kmod2);
          const double corr = lw != 0.0 ? tanh(kmod * lw) : 1.0;
          amp = 1.0 / sqrt(kmod * kmod2 * (kmod + kc * corr));
        } else {
          amp = 1.0 / (mkx * mkx + mky * mky);
        }
        if (edge) {
          Wxr = sqrt(2.0) * prefactor * amp * (mky * Rn[index]);
          Wyr = sqrt(2.0) * prefactor * amp * ((-mkx) * Rn[index]);
        } else {
          Wxr = prefactor * amp * (mky * Rn[index]);
          Wyr = prefactor * amp * ((-mkx) * Rn[index]);
          Wxi = prefactor * amp * (mky * Rn[nModes * 2 + index]);
          Wyi = prefactor * amp * ((-mkx) * Rn[nModes * 2 + index]);
        }
      }
    }
    if ((fx < 0) || (fx == 0 && fy < 0)) {
      Wxi = -Wxi;
      Wyi = -Wyi;
    }
    R.z64[i] = make_double2(oxr + Wxr, oxi + Wxi);
    R.z64[nc + i] = make_double2(oyr + Wyr, oyi + Wyi);
  }
}

// ------------------------------------------------------- particle update --
// q_out = q + dx dy h J(q_at) v (src/quasi2DFunctions.cu:681-760): stage 1
// interpolates at q and writes q^{n+1/2} with h = dt/2 (predictor-corrector)
// or q^{n+1} with h = dt (forward Euler); stage 2 interpolates at q^{n+1/2}
// and writes q^{n+1} with h = dt.
template <bool ONE>
__global__ void k_q2_update(FSL_KARGS, int stage) {
  FSL_REP_FLAT(KIND_T1);
  const int i = blk * blockDim.x + threadIdx.x;
  const int np = P.np;
  if (i >= np || (stage == 2 && !P.q2_pc)) return;
  const double* at = stage == 2 ? R.qp : R.q;
  const double rx = at[i], ry = at[np + i];
  const int mx = P.mx, my = P.my, w = P.q2_kw;
  const int kx = cellidx(minimage(rx, P.invlx, P.lx), P.invdx, mx);
  const int ky = cellidx(minimage(ry, P.invly, P.ly), P.invdy, my);
  const double* vx = R.v64;
  const double* vy = R.v64 + P.nc;
  double ux = 0.0, uy = 0.0;
  for (int ix = -w; ix <= w; ++ix) {
    const int kxn = node_wrap(kx, ix, mx);
    const double dxr = node_dist(rx, kxn, P.lx, mx, P.invlx);
    for (int iy = -w; iy <= w; ++iy) {
      const int kyn = node_wrap(ky, iy, my);
      const double dyr = node_dist(ry, kyn, P.ly, my, P.invly);
      const double g = gauss2d(dxr * dxr + dyr * dyr, P.q2_var);
      ux += g * vx[kxn + kyn * mx];
      uy += g * vy[kxn + kyn * mx];
    }
  }
  const double vol = P.dx * P.dy;
  const double h = (stage == 1 && P.q2_pc) ? 0.5 * P.dt : P.dt;
  double* out = (stage == 1 && P.q2_pc) ? R.qp : R.q;
  const double nx = R.q[i] + vol * ux * h, ny = R.q[np + i] + vol * uy * h;
  if (!isfinite(nx) || !isfinite(ny)) set_err(R.err, 2);
  out[i] = nx;
  out[np + i] = ny;
  if (stage == 1 && P.q2_pc) out[2 * (size_t)np + i] = R.q[2 * (size_t)np + i];
}

}  // namespace

// ------------------------------------------------------------ launchers --
void launch_q2_forces(const Batch& B, cudaStream_t s) {
  if (B.max_np == 0) return;
  FSL_GO(k_q2_forces, part_blocks(B, KIND_T1), kPartThreads, 0, s, B);
}

void launch_q2_field(const Batch& B, cudaStream_t s, Prof* prof) {
  const int tb = 256;
  unsigned bc = blocks_for((long)2 * B.nc, tb);
  const unsigned cap = (unsigned)((148 * 16 + B.nrep - 1) / B.nrep);
  if (bc > cap) bc = cap < 1 ? 1 : cap;
  if (prof) prof->mark(s, "q2_spread");
  FSL_GO(k_q2_zero, dim3(bc, B.nrep), tb, 0, s, B);
  if (B.max_np > 0) FSL_GO(k_q2_spread, part_blocks(B, KIND_T1), kPartThreads, 0, s, B);
  FSL_GO(k_q2_shear, dim3(bc, B.nrep), tb, 0, s, B);
}

void launch_q2_solve(const Batch& B, cudaStream_t s, Prof* prof) {
  const int tb = 256;
  unsigned bc = blocks_for((long)B.nc, tb);
  const unsigned cap = (unsigned)((148 * 16 + B.nrep - 1) / B.nrep);
  if (bc > cap) bc = cap < 1 ? 1 : cap;
  if (prof) prof->mark(s, "q2_fft");
  launch_fft64_2d(B, -1, s);
  if (prof) prof->mark(s, "q2_fourier");
  FSL_GO(k_q2_fourier, dim3(bc, B.nrep), tb, 0, s, B);
  if (prof) prof->mark(s, "q2_fft");
  launch_fft64_2d(B, +1, s);
}

void launch_q2_update(const Batch& B, int stage, cudaStream_t s) {
  if (B.max_np == 0) return;
  FSL_GO(k_q2_update, part_blocks(B, KIND_T1), kPartThreads, 0, s, B, stage);
}

}  // namespace fsl
