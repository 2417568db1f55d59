// fsl_fp64.cu -- the FP64 form of the fluid side (FSL_PRECISION_FP64).
//
// The step of the FP32 kernels with every fluid quantity in double: the
// noise (Box-Muller in FP64 on the same Philox words), spreading with FP64
// atomics, W, the FFT-based Stokes solve and the interpolation.  fluam itself
// is FP64 throughout, so this form carries the reference's own arithmetic on
// the GPU; it is the third form of the precision study and is written for
// clarity over speed: one thread per particle and component for the particle
// side, shared-memory Stockham lines (any 2,3,5,7,11-smooth length) with the
// twiddles evaluated in place for the FFTs.  The cell list and the forces
// are the shared FP64 kernels of fsl_particles.cu.
#include "fsl_internal.cuh"

namespace fsl {

namespace {

unsigned blocks_for(long work, int tb) { return (unsigned)((work + tb - 1) / tb); }

// ------------------------------------------------------------------ noise ---
// Normal deviates 4b .. 4b+3 of draw t: the Philox words and uniforms of
// philox_normal4, radius sqrt(-2 ln u) and angle 2 pi u in FP64.
__device__ __forceinline__ void philox_normal4_f64(uint64_t seed, uint64_t t, uint64_t b,
                                                   double2& lo, double2& hi) {
  uint4 c = make_uint4((uint32_t)b, (uint32_t)(b >> 32), (uint32_t)t, (uint32_t)(t >> 32));
  uint4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double s24 = 5.9604644775390625e-08;  // 2^-24
  const double u0 = (double)(2u * (r.x >> 9) + 1u) * s24;
  const double u1 = (double)(2u * (r.y >> 9) + 1u) * s24;
  const double u2 = (double)(2u * (r.z >> 9) + 1u) * s24;
  const double u3 = (double)(2u * (r.w >> 9) + 1u) * s24;
  const double twopi = 6.283185307179586476925286766559;
  const double ra = sqrt(-2.0 * log(u0)), rb = sqrt(-2.0 * log(u2));
  double sa, ca, sb, cb;
  sincos(twopi * u1, &sa, &ca);
  sincos(twopi * u3, &sb, &cb);
  lo = make_double2(ra * ca, ra * sa);
  hi = make_double2(rb * cb, rb * sb);
}

template <bool ONE>
__global__ void k_noise64(FSL_KARGS) {
  FSL_REP_AT(blockIdx.y);
  const uint64_t t = *R.t;
  const uint64_t nb = (P.noise_n + 3) >> 2;
  double2* out = reinterpret_cast<double2*>(R.noise64);
  for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nb;
       b += (uint64_t)gridDim.x * blockDim.x) {
    double2 lo, hi;
    philox_normal4_f64(P.seed, t, b, lo, hi);
    out[2 * b] = lo;
    out[2 * b + 1] = hi;
  }
}

// --------------------------------------------------------------- stencils ---
// 3-point kernel of src/deltaGPU.cu:57-68, with its single-precision square
// root of a double argument.
__device__ __forceinline__ double delta3d(double x) {
  x = fabs(x);
  if (x > 1.5) return 0.0;
  if (x < 0.5) return (1. + (double)sqrtf((float)(1. - 3. * x * x))) / 3.;
  return (5. - 3. * x - (double)sqrtf((float)(1. - 3. * (1. - x) * (1. - x)))) / 6.;
}

// 4-point kernel (Peskin, Acta Numerica 2002), the form of delta4f in FP64.
__device__ __forceinline__ double delta4d(double x) {
  x = fabs(x);
  if (x >= 2.0) return 0.0;
  if (x <= 1.0) return (3. - 2. * x + sqrt(1. + 4. * x - 4. * x * x)) / 8.;
  return (5. - 2. * x - sqrt(fmax(-7. + 12. * x - 4. * x * x, 0.0))) / 8.;
}

struct Stencil64 {
  int j0[3];
  double w[3][4];
};

// Stencil of component comp: the node choice of stencil_node (posc) and the
// weights in FP64 (posw).
__device__ __forceinline__ void stencil64(const Params& P, int comp, const double posc[3],
                                          const double posw[3], Stencil64& st) {
  const int m[3] = {P.mx, P.my, P.mz};
  const double h[3] = {P.dx, P.dy, P.dz};
  const double invd[3] = {P.invdx, P.invdy, P.invdz};
  const double L[3] = {P.lx, P.ly, P.lz};
  const double invL[3] = {P.invlx, P.invly, P.invlz};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double off = (d == comp) ? __dmul_rn(0.5, h[d]) : 0.0;
    if (P.kernel == 3) {
      double r = minimage(__dsub_rn(posc[d], off), invL[d], L[d]);
      st.j0[d] = wrap_add(cellidx(r, invd[d], m[d]), -1, m[d]);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        int j = wrap_add(st.j0[d], k, m[d]);
        double node = ((double)j + 0.5) * h[d] - 0.5 * L[d];
        double rr = minimage((posw[d] - node) - off, invL[d], L[d]);
        st.w[d][k] = delta3d(rr * invd[d]);
      }
      st.w[d][3] = 0.0;
    } else {
      double r = minimage(__dsub_rn(__dsub_rn(posc[d], off), __dmul_rn(0.5, h[d])), invL[d], L[d]);
      st.j0[d] = wrap_add(cellidx(r, invd[d], m[d]), -1, m[d]);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        int j = (st.j0[d] + k) % m[d];
        double node = ((double)j + 0.5) * h[d] - 0.5 * L[d] + off;
        st.w[d][k] = delta4d(minimage(posw[d] - node, invL[d], L[d]) * invd[d]);
      }
    }
  }
}

template <int KN>
__device__ __forceinline__ void spread64_one(const Params& P, int comp, const double posc[3],
                                             const double posw[3], double val,
                                             double* __restrict__ g) {
  Stencil64 st;
  stencil64(P, comp, posc, posw, st);
  double* gc = g + (size_t)comp * P.nc;
#pragma unroll
  for (int c = 0; c < KN; ++c) {
    const int z = (st.j0[2] + c) % P.mz;
#pragma unroll
    for (int b = 0; b < KN; ++b) {
      const int y = (st.j0[1] + b) % P.my;
      const double wyz = st.w[1][b] * st.w[2][c] * val;
      const size_t row = (size_t)P.mx * (y + (size_t)P.my * z);
#pragma unroll
      for (int a = 0; a < KN; ++a) {
        const double v = st.w[0][a] * wyz;
        if (v != 0.0) atomicAdd(gc + row + (st.j0[0] + a) % P.mx, v);
      }
    }
  }
}

// ---------------------------------------------------------------- spread ---
// Eight threads per particle: thread s < 3 spreads component s of the force,
// 3 <= s < 6 (drift modes) component s-3 of the RFD drift (both signs).
// drift: 0 F at q; 1 F at q^{n+1/2} + drift; 2 F at q + drift.  The field is
// the FP64 view of the 8-byte spread buffer; W's build divides by dV.
template <bool ONE, int KN>
__global__ void k_spread64(FSL_KARGS, int drift) {
  FSL_REP_FLAT(KIND_T8);
  const long t = blk * (long)blockDim.x + threadIdx.x;
  const int i = (int)(t >> 3), sub = (int)(t & 7);
  const int np = P.np;
  if (i >= np || sub >= (drift ? 6 : 3)) return;
  double* g = reinterpret_cast<double*>(R.grid);
  if (sub < 3) {
    const double* qf = drift == 1 ? R.qp : R.q;
    const double pos[3] = {qf[i], qf[np + i], qf[2 * (size_t)np + i]};
    spread64_one<KN>(P, sub, pos, pos, R.F[(size_t)sub * np + i], g);
    return;
  }
  const int comp = sub - 3;
  const size_t wb = (size_t)6 * P.nc;
  const double W[3] = {R.noise64[wb + i], R.noise64[wb + np + i], R.noise64[wb + 2 * (size_t)np + i]};
  const double pos[3] = {R.q[i], R.q[np + i], R.q[2 * (size_t)np + i]};
  double pp[3], pm[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    pp[d] = pos[d] + 0.5 * kRfdDelta * W[d];
    pm[d] = pos[d] - 0.5 * kRfdDelta * W[d];
  }
  const double vp = (P.kT / kRfdDelta) * W[comp], vm = (P.kT / kRfdDelta) * -1 * W[comp];
  // reference mode: nodes from the displaced position, weights at q
  spread64_one<KN>(P, comp, pp, P.rfd == 1 ? pp : pos, vp, g);
  spread64_one<KN>(P, comp, pm, P.rfd == 1 ? pm : pos, vm, g);
}

// ------------------------------------------------------------------- W ---
// W = f / dV + nfac div(Sigma) per cell (the formulas of k_wbuild in FP64),
// written as the real part of the spectrum buffer; the spread field is
// cleared behind the read.
template <bool ONE>
__global__ void k_wbuild64(FSL_KARGS, int nsets, double nfac) {
  FSL_REP_AT(blockIdx.y);
  const size_t nc = (size_t)P.nc;
  const int mx = P.mx, my = P.my, mz = P.mz;
  const double inv_dV = 1.0 / P.dV;
  const double f1 = nfac * P.fact1, f4 = nfac * P.fact4;
  const double a1x = P.invdx * f1, a1y = P.invdy * f1, a1z = P.invdz * f1;
  const double a4x = P.invdx * f4, a4y = P.invdy * f4, a4z = P.invdz * f4;
  double* g = reinterpret_cast<double*>(R.grid);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nc;
       i += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % mx), r = (int)(i / mx);
    const int y = r % my, z = r / my;
    const int xm = x == 0 ? mx - 1 : x - 1, xp = x == mx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? my - 1 : y - 1, yp = y == my - 1 ? 0 : y + 1;
    const int zm = z == 0 ? mz - 1 : z - 1, zp = z == mz - 1 ? 0 : z + 1;
    const size_t rowyz = (size_t)mx * (y + (size_t)my * z);
    const size_t v0 = x + (size_t)mx * (y + (size_t)my * zm), v1 = x + (size_t)mx * (ym + (size_t)my * z),
                 v2 = xm + rowyz, v3 = xp + rowyz, v4 = x + (size_t)mx * (yp + (size_t)my * z),
                 v5 = x + (size_t)mx * (y + (size_t)my * zp);
    double w[3] = {g[i] * inv_dV, g[nc + i] * inv_dV, g[2 * nc + i] * inv_dV};
    for (int set = 0; set < nsets; ++set) {
      const double* d = R.noise64 + (set ? (size_t)6 * nc + (size_t)9 * P.np : 0);
      w[0] += a1x * (d[v3] - d[i]) + a4y * (d[nc + i] - d[nc + v1]) + a4z * (d[2 * nc + i] - d[2 * nc + v0]);
      w[1] += a1y * (d[3 * nc + v4] - d[3 * nc + i]) + a4x * (d[nc + i] - d[nc + v2]) +
              a4z * (d[4 * nc + i] - d[4 * nc + v0]);
      w[2] += a1z * (d[5 * nc + v5] - d[5 * nc + i]) + a4x * (d[2 * nc + i] - d[2 * nc + v2]) +
              a4y * (d[4 * nc + i] - d[4 * nc + v1]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      R.z64[c * nc + i] = make_double2(w[c], 0.0);
      g[c * nc + i] = 0.0;
    }
  }
}

// ------------------------------------------------------------------- FFT ---
// Complex lines of length n along one axis of the three-component array,
// transformed in shared memory by the Stockham autosort algorithm
// (Govindaraju et al., SC'08) with mixed radices 4, 2, 3, 5, 7, 11: stage
// with radix p and span Ns reads v_r = X[j + r n/p], twiddles v_r by
// exp(dir 2 pi i r (j mod Ns) / (Ns p)), a p-point DFT, and writes
// Y[(j / Ns) Ns p + (j mod Ns) + r Ns].  Unnormalised, dir -1 forward.
struct Radix64 {
  int n, nf, f[12];
};

Radix64 radices(int n) {
  Radix64 R{};
  R.n = n;
  while (n % 4 == 0) { R.f[R.nf++] = 4; n /= 4; }
  const int ps[5] = {2, 3, 5, 7, 11};
  for (int p : ps)
    while (n % p == 0) { R.f[R.nf++] = p; n /= p; }
  return R;
}

template <int Pr>
__device__ __forceinline__ void dft64(double2 (&v)[Pr], int dir) {
  if constexpr (Pr == 2) {
    double2 a = v[0], b = v[1];
    v[0] = make_double2(a.x + b.x, a.y + b.y);
    v[1] = make_double2(a.x - b.x, a.y - b.y);
  } else if constexpr (Pr == 4) {
    const double2 a0 = make_double2(v[0].x + v[2].x, v[0].y + v[2].y);
    const double2 a1 = make_double2(v[0].x - v[2].x, v[0].y - v[2].y);
    const double2 b0 = make_double2(v[1].x + v[3].x, v[1].y + v[3].y);
    const double2 b1 = make_double2(v[1].x - v[3].x, v[1].y - v[3].y);
    // multiply b1 by dir * i
    const double2 ib1 = make_double2(-dir * b1.y, dir * b1.x);
    v[0] = make_double2(a0.x + b0.x, a0.y + b0.y);
    v[2] = make_double2(a0.x - b0.x, a0.y - b0.y);
    v[1] = make_double2(a1.x + ib1.x, a1.y + ib1.y);
    v[3] = make_double2(a1.x - ib1.x, a1.y - ib1.y);
  } else {
    double2 w[Pr], o[Pr];  // w[k] = exp(dir 2 pi i k / Pr)
#pragma unroll
    for (int k = 0; k < Pr; ++k) sincospi((double)(2 * k) / Pr * dir, &w[k].y, &w[k].x);
#pragma unroll
    for (int q = 0; q < Pr; ++q) {
      double sx = 0.0, sy = 0.0;
#pragma unroll
      for (int r = 0; r < Pr; ++r) {
        const double2 t = w[(r * q) % Pr];
        sx += v[r].x * t.x - v[r].y * t.y;
        sy += v[r].x * t.y + v[r].y * t.x;
      }
      o[q] = make_double2(sx, sy);
    }
#pragma unroll
    for (int q = 0; q < Pr; ++q) v[q] = o[q];
  }
}

template <int Pr>
__device__ void stage64(const double2* __restrict__ X, double2* __restrict__ Y, int n, int Ns,
                        int nl, int dir) {
  const int nb = n / Pr;
  for (int t = threadIdx.x; t < nl * nb; t += blockDim.x) {
    const int l = t / nb, j = t - l * nb;
    const double2* x = X + (size_t)l * n;
    double2* y = Y + (size_t)l * n;
    const int k = j % Ns;
    double2 v[Pr];
#pragma unroll
    for (int r = 0; r < Pr; ++r) v[r] = x[j + r * nb];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < Pr; ++r) {
        double s, c;
        sincospi((double)(2 * r * k) / (double)(Ns * Pr) * dir, &s, &c);
        v[r] = make_double2(v[r].x * c - v[r].y * s, v[r].x * s + v[r].y * c);
      }
    }
    dft64<Pr>(v, dir);
    const int d = (j / Ns) * Ns * Pr + k;
#pragma unroll
    for (int r = 0; r < Pr; ++r) y[d + r * Ns] = v[r];
  }
}

constexpr int kF64Threads = 256;
constexpr int kF64Elems = 1024;  // lines x length per block: 2 x 16 KB buffers

// Lines of one block: axis 0 takes nl consecutive rows (contiguous);
// axes 1 and 2 take nl consecutive x at one (comp, other index), element
// stride mx or mx my; ncomp field components.  to_real: the last inverse
// pass stores Re / nc to v64.
template <bool ONE>
__global__ void __launch_bounds__(kF64Threads) k_fft64(FSL_KARGS, int axis, const Radix64 rad,
                                                       int dir, int to_real, int ncomp) {
  FSL_REP_AT(blockIdx.y);
  __shared__ double2 sA[kF64Elems], sB[kF64Elems];
  const int n = rad.n;
  const int mx = P.mx, my = P.my, mz = P.mz;
  const size_t nc = (size_t)P.nc;
  const int nl = kF64Elems / n < 1 ? 1 : (kF64Elems / n > 32 ? 32 : kF64Elems / n);
  size_t base;
  size_t estride, lstride;
  int nvalid;
  if (axis == 0) {
    const long nrows = (long)ncomp * my * mz;
    const long r0 = (long)blockIdx.x * nl;
    if (r0 >= nrows) return;
    base = (size_t)r0 * mx;
    estride = 1;
    lstride = (size_t)mx;
    nvalid = (int)min((long)nl, nrows - r0);
  } else {
    const int gx = (mx + nl - 1) / nl;
    const int other = axis == 1 ? mz : my;
    const long b = blockIdx.x;
    if (b >= (long)ncomp * other * gx) return;
    const int xg = (int)(b % gx);
    const long rest = b / gx;
    const int o = (int)(rest % other), comp = (int)(rest / other);
    const int x0 = xg * nl;
    base = comp * nc + x0 + (axis == 1 ? (size_t)mx * my * o : (size_t)mx * o);
    estride = axis == 1 ? (size_t)mx : (size_t)mx * my;
    lstride = 1;
    nvalid = min(nl, mx - x0);
  }
  double2* Z = R.z64;
  // load: consecutive threads take consecutive addresses
  for (int t = threadIdx.x; t < nl * n; t += blockDim.x) {
    int l, j;
    if (axis == 0) { l = t / n; j = t - l * n; }
    else { j = t / nl; l = t - j * nl; }
    sA[l * n + j] = l < nvalid ? Z[base + l * lstride + j * estride] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double2* X = sA;
  double2* Y = sB;
  int Ns = 1;
  for (int s = 0; s < rad.nf; ++s) {
    const int p = rad.f[s];
    switch (p) {
      case 4: stage64<4>(X, Y, n, Ns, nl, dir); break;
      case 2: stage64<2>(X, Y, n, Ns, nl, dir); break;
      case 3: stage64<3>(X, Y, n, Ns, nl, dir); break;
      case 5: stage64<5>(X, Y, n, Ns, nl, dir); break;
      case 7: stage64<7>(X, Y, n, Ns, nl, dir); break;
      default: stage64<11>(X, Y, n, Ns, nl, dir); break;
    }
    __syncthreads();
    double2* tmp = X;
    X = Y;
    Y = tmp;
    Ns *= p;
  }
  const double inv_nc = 1.0 / (double)nc;
  for (int t = threadIdx.x; t < nl * n; t += blockDim.x) {
    int l, j;
    if (axis == 0) { l = t / n; j = t - l * n; }
    else { j = t / nl; l = t - j * nl; }
    if (l >= nvalid) continue;
    const size_t a = base + l * lstride + j * estride;
    if (to_real) R.v64[a] = X[l * n + j].x * inv_nc;
    else Z[a] = X[l * n + j];
  }
}

// Fourier-space solve per mode (src/stokesLimitFunctions.cu:2399-2451 with
// the staggered shifts of src/realToComplex.cu:263-303 and the tables of
// src/initializePrefactorFourierSpace.cu:39-69, evaluated in place).
template <bool ONE>
__global__ void k_solve64(FSL_KARGS) {
  FSL_REP_AT(blockIdx.y);
  const int mx = P.mx, my = P.my, mz = P.mz;
  const size_t nc = (size_t)P.nc;
  const double pi = 3.141592653589793238462643383280;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nc;
       i += (size_t)gridDim.x * blockDim.x) {
    const int kx = (int)(i % mx), r = (int)(i / mx);
    const int ky = r % my, kz = r / my;
    const int kk[3] = {kx, ky, kz};
    const int m[3] = {mx, my, mz};
    const double invd[3] = {P.invdx, P.invdy, P.invdz};
    double c[3], sn[3], gk[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double arg = pi * kk[a] / (double)m[a];
      sincos(arg, &sn[a], &c[a]);
      gk[a] = 2 * invd[a] * sn[a];
    }
    double2 W[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double2 z = R.z64[a * nc + i];
      // shift -1: W (cos - i sin)
      W[a] = make_double2(z.x * c[a] + z.y * sn[a], z.y * c[a] - z.x * sn[a]);
    }
    double2 V[3];
    if (i == 0) {
      V[0] = V[1] = V[2] = make_double2(0.0, 0.0);
    } else {
      const double L = -(gk[0] * gk[0]) - (gk[1] * gk[1]) - (gk[2] * gk[2]);
      const double den = -P.eta * L;
      const double GWr = gk[0] * W[0].x + gk[1] * W[1].x + gk[2] * W[2].x;
      const double GWi = gk[0] * W[0].y + gk[1] * W[1].y + gk[2] * W[2].y;
#pragma unroll
      for (int a = 0; a < 3; ++a)
        V[a] = make_double2((W[a].x + gk[a] * GWr / L) / den, (W[a].y + gk[a] * GWi / L) / den);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)  // shift +1: V (cos + i sin)
      R.z64[a * nc + i] = make_double2(V[a].x * c[a] - V[a].y * sn[a], V[a].y * c[a] + V[a].x * sn[a]);
  }
}

// ------------------------------------------------------ interpolation ---
// Eight threads per particle, thread s < 3 interpolates component s and
// updates that coordinate: stage 1 q^{n+1/2} = q^n + dt/2 J(q^n) v, stage 2
// q^{n+1} = q^n + dt J(q^{n+1/2}) v, each with the extraMobility terms
// (src/stokesLimitFunctions.cu:2646-2650, 3676-3681).
template <bool ONE, int KN>
__global__ void k_interp_update64(FSL_KARGS, int stage) {
  FSL_REP_FLAT(KIND_T8);
  const long t = blk * (long)blockDim.x + threadIdx.x;
  const int i = (int)(t >> 3), comp = (int)(t & 7);
  const int np = P.np;
  if (i >= np || comp >= 3) return;
  const double* qpos = stage == 1 ? R.q : R.qp;
  double* qout = stage == 1 ? R.qp : R.q;
  const double pos[3] = {qpos[i], qpos[np + i], qpos[2 * (size_t)np + i]};
  Stencil64 st;
  stencil64(P, comp, pos, pos, st);
  const double* vc = R.v64 + (size_t)comp * P.nc;
  double u = 0.0;
#pragma unroll
  for (int a = 0; a < KN; ++a) {
    const int x = (st.j0[0] + a) % P.mx;
#pragma unroll
    for (int b = 0; b < KN; ++b) {
      const int y = (st.j0[1] + b) % P.my;
#pragma unroll
      for (int c = 0; c < KN; ++c) {
        const int z = (st.j0[2] + c) % P.mz;
        u += st.w[0][a] * st.w[1][b] * st.w[2][c] * vc[x + (size_t)P.mx * (y + (size_t)P.my * z)];
      }
    }
  }
  const size_t k = (size_t)comp * np + i;
  const double h = stage == 1 ? 0.5 * P.dt : P.dt;
  double r = R.q[k] + h * u;
  if (P.has_extra) {
    const size_t nb = (size_t)6 * P.nc + (size_t)(3 + comp) * np + i;
    double xi = R.noise64[nb];
    if (stage == 2) xi += R.noise64[nb + (size_t)3 * np];
    r += h * P.extra_mob * R.F[k] + P.fact2 * xi;
  }
  if (!isfinite(r)) set_err(R.err, 2);
  qout[k] = r;
}

}  // namespace

// ---------------------------------------------------------------- launchers
void launch_noise64(const Batch& B, cudaStream_t s) {
  const int tb = 256;
  const uint64_t nb = (B.max_noise_n + 3) / 4;
  unsigned bx = blocks_for((long)nb, tb);
  const unsigned cap = (unsigned)((148 * 16 + B.nrep - 1) / B.nrep);
  if (bx > cap) bx = cap < 1 ? 1 : cap;
  FSL_GO(k_noise64, dim3(bx, B.nrep), tb, 0, s, B);
}

void launch_spread64(const Batch& B, int drift, cudaStream_t s) {
  if (B.max_np == 0) return;
  const unsigned g = part_blocks(B, KIND_T8);
  if (B.kernel == 4)
    FSL_GO_T(k_spread64, 4, g, kPartThreads, 0, s, B, drift);
  else
    FSL_GO_T(k_spread64, 3, g, kPartThreads, 0, s, B, drift);
}

void launch_interp_update64(const Batch& B, int stage, cudaStream_t s) {
  if (B.max_np == 0) return;
  const unsigned g = part_blocks(B, KIND_T8);
  if (B.kernel == 4)
    FSL_GO_T(k_interp_update64, 4, g, kPartThreads, 0, s, B, stage);
  else
    FSL_GO_T(k_interp_update64, 3, g, kPartThreads, 0, s, B, stage);
}

// The line passes of a forward (dir -1: x, y[, z]) or inverse (dir +1:
// [z,] y, x, the x pass storing Re / nc) transform of ncomp components over
// the first naxes axes.
static void fft64_passes(const Batch& B, int ncomp, int naxes, int dir, cudaStream_t s,
                         int to_real = 1) {
  const int m[3] = {B.mx, B.my, B.mz};
  Radix64 rad[3];
  unsigned gb[3];
  for (int a = 0; a < naxes; ++a) {
    rad[a] = radices(m[a]);
    const int n = m[a];
    const int nl = kF64Elems / n < 1 ? 1 : (kF64Elems / n > 32 ? 32 : kF64Elems / n);
    if (a == 0) gb[a] = (unsigned)(((long)ncomp * B.my * B.mz + nl - 1) / nl);
    else gb[a] = (unsigned)((long)ncomp * (a == 1 ? B.mz : B.my) * ((B.mx + nl - 1) / nl));
  }
  if (dir < 0) {
    for (int a = 0; a < naxes; ++a)
      FSL_GO(k_fft64, dim3(gb[a], B.nrep), kF64Threads, 0, s, B, a, rad[a], -1, 0, ncomp);
  } else {
    for (int a = naxes - 1; a >= 0; --a)
      FSL_GO(k_fft64, dim3(gb[a], B.nrep), kF64Threads, 0, s, B, a, rad[a], +1, a == 0 ? to_real : 0,
             ncomp);
  }
}

void launch_solve64(const Batch& B, int nsets, double nfac, cudaStream_t s, Prof* prof) {
  const int tb = 256;
  unsigned bc = blocks_for((long)B.nc, tb);
  const unsigned cap = (unsigned)((148 * 16 + B.nrep - 1) / B.nrep);
  if (bc > cap) bc = cap < 1 ? 1 : cap;
  if (prof) prof->mark(s, "wbuild64");
  FSL_GO(k_wbuild64, dim3(bc, B.nrep), tb, 0, s, B, nsets, nfac);
  if (prof) prof->mark(s, "fft64");
  fft64_passes(B, 3, 3, -1, s);
  if (prof) prof->mark(s, "solve64");
  FSL_GO(k_solve64, dim3(bc, B.nrep), tb, 0, s, B);
  if (prof) prof->mark(s, "fft64");
  fft64_passes(B, 3, 3, +1, s);
  if (prof) prof->count(1 + 3 + 1 + 3);
}

void launch_fft64_2d(const Batch& B, int dir, cudaStream_t s) { fft64_passes(B, 2, 2, dir, s); }

void launch_fft64_3d(const Batch& B, int dir, int to_real, cudaStream_t s) {
  fft64_passes(B, 3, 3, dir, s, to_real);
}

}  // namespace fsl
