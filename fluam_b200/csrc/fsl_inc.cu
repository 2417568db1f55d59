// fsl_inc.cu -- the incompressible fluctuating fluid (FSL_SCHEME_INCOMPRESSIBLE).
//
// The solver of keyword incompressible (src/runSchemeIncompressible.cu:
// 20-155), FP64 as the reference: staggered velocities u (Rep::v64), a
// Crank-Nicolson viscous term and a midpoint advection in two substeps that
// share one noise draw, each substep a W build in real space, a forward FFT,
// the shifted Crank-Nicolson solve with the divergence-free projection per
// mode, and an inverse FFT.  The prediction u^{n+1/2} of the first substep
// lives in the 8-byte spread buffer (Rep::grid, unused by this scheme).  The
// FFT passes are those of the FP64 form (fsl_fp64.cu).
#include "fsl_internal.cuh"

namespace fsl {

namespace {

unsigned blocks_for(long work, int tb) { return (unsigned)((work + tb - 1) / tb); }

__device__ __forceinline__ int wrapi(int j, int m) { return j < 0 ? j + m : (j >= m ? j - m : j); }

// W = u + dt/2 (eta/rho) L u - (dt/4) A(a) + div(Sigma) per cell, the
// advection A of field a (u, or the prediction in the second substep),
// src/kernelConstructW.cu:32-265 and 266-521; the random stress is the
// traceless symmetric tensor with layout XX, XY, XZ, YY, YZ, ZZ.
template <bool ONE>
__global__ void k_inc_w(FSL_KARGS, int second) {
  FSL_REP_AT(blockIdx.y);
  const int mx = P.mx, my = P.my, mz = P.mz, nc = P.nc;
  const double* ux = R.v64;
  const double* uy = R.v64 + nc;
  const double* uz = R.v64 + 2 * (size_t)nc;
  const double* a = second ? reinterpret_cast<const double*>(R.grid) : R.v64;
  const double* ax = a;
  const double* ay = a + nc;
  const double* az = a + 2 * (size_t)nc;
  const double* Rn = R.noise64;
  const double idx = P.invdx, idy = P.invdy, idz = P.invdz, dt = P.dt;
  const double nu = P.eta / P.rho, f1 = P.fact1, f4 = P.fact4;
  const size_t n = (size_t)nc;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
    const int x = i % mx, y = (i / mx) % my, z = i / (mx * my);
    auto at = [&](int dx, int dy, int dz) {
      return wrapi(x + dx, mx) + mx * (wrapi(y + dy, my) + my * wrapi(z + dz, mz));
    };
    const int v0 = at(0, 0, -1), v1 = at(0, -1, 0), v2 = at(-1, 0, 0), v3 = at(1, 0, 0),
              v4 = at(0, 1, 0), v5 = at(0, 0, 1);
    const int pxmy = at(1, -1, 0), pxmz = at(1, 0, -1), mxpy = at(-1, 1, 0), mxpz = at(-1, 0, 1),
              pymz = at(0, 1, -1), mypz = at(0, -1, 1);
    double wx = idx * idx * (ux[v3] - 2 * ux[i] + ux[v2]);
    wx += idy * idy * (ux[v4] - 2 * ux[i] + ux[v1]);
    wx += idz * idz * (ux[v5] - 2 * ux[i] + ux[v0]);
    wx = 0.5 * dt * nu * wx;
    double wy = idx * idx * (uy[v3] - 2 * uy[i] + uy[v2]);
    wy += idy * idy * (uy[v4] - 2 * uy[i] + uy[v1]);
    wy += idz * idz * (uy[v5] - 2 * uy[i] + uy[v0]);
    wy = 0.5 * dt * nu * wy;
    double wz = idx * idx * (uz[v3] - 2 * uz[i] + uz[v2]);
    wz += idy * idy * (uz[v4] - 2 * uz[i] + uz[v1]);
    wz += idz * idz * (uz[v5] - 2 * uz[i] + uz[v0]);
    wz = 0.5 * dt * nu * wz;
    wx += ux[i];
    wy += uy[i];
    wz += uz[i];
    double advX = idx * ((ax[v3] + ax[i]) * (ax[v3] + ax[i]) - (ax[i] + ax[v2]) * (ax[i] + ax[v2]));
    advX += idy * ((ax[v4] + ax[i]) * (ay[v3] + ay[i]) - (ax[i] + ax[v1]) * (ay[pxmy] + ay[v1]));
    advX += idz * ((ax[v5] + ax[i]) * (az[v3] + az[i]) - (ax[i] + ax[v0]) * (az[pxmz] + az[v0]));
    advX = 0.25 * dt * advX;
    double advY = idx * ((ay[v3] + ay[i]) * (ax[v4] + ax[i]) - (ay[i] + ay[v2]) * (ax[mxpy] + ax[v2]));
    advY += idy * ((ay[v4] + ay[i]) * (ay[v4] + ay[i]) - (ay[i] + ay[v1]) * (ay[i] + ay[v1]));
    advY += idz * ((ay[v5] + ay[i]) * (az[v4] + az[i]) - (ay[i] + ay[v0]) * (az[pymz] + az[v0]));
    advY = 0.25 * dt * advY;
    double advZ = idx * ((az[v3] + az[i]) * (ax[v5] + ax[i]) - (az[i] + az[v2]) * (ax[mxpz] + ax[v2]));
    advZ += idy * ((az[v4] + az[i]) * (ay[v5] + ay[i]) - (az[i] + az[v1]) * (ay[mypz] + ay[v1]));
    advZ += idz * ((az[v5] + az[i]) * (az[v5] + az[i]) - (az[i] + az[v0]) * (az[i] + az[v0]));
    advZ = 0.25 * dt * advZ;
    wx -= advX;
    wy -= advY;
    wz -= advZ;
    auto trace = [&](int c) { return Rn[c] + Rn[c + 3 * n] + Rn[c + 5 * n]; };
    wx += idx * f1 * (Rn[v3] - trace(v3) / 3.);
    wy += idy * f1 * (Rn[v4 + 3 * n] - trace(v4) / 3.);
    wz += idz * f1 * (Rn[v5 + 5 * n] - trace(v5) / 3.);
    wx += idy * f4 * Rn[i + n];
    wy += idx * f4 * Rn[i + n];
    wx += idz * f4 * Rn[i + 2 * n];
    wz += idx * f4 * Rn[i + 2 * n];
    wy += idz * f4 * Rn[i + 4 * n];
    wz += idy * f4 * Rn[i + 4 * n];
    const double tr = trace(i);
    wx -= idx * f1 * (Rn[i] - tr / 3.);
    wy -= idy * f1 * (Rn[i + 3 * n] - tr / 3.);
    wz -= idz * f1 * (Rn[i + 5 * n] - tr / 3.);
    wx -= idy * f4 * Rn[v1 + n];
    wx -= idz * f4 * Rn[v0 + 2 * n];
    wy -= idx * f4 * Rn[v2 + n];
    wy -= idz * f4 * Rn[v0 + 4 * n];
    wz -= idx * f4 * Rn[v2 + 2 * n];
    wz -= idy * f4 * Rn[v1 + 4 * n];
    R.z64[i] = make_double2(wx, 0.0);
    R.z64[n + i] = make_double2(wy, 0.0);
    R.z64[2 * n + i] = make_double2(wz, 0.0);
  }
}

// Per mode: shift(-1), the Crank-Nicolson solve with the projection
// (src/kernelUpdateVIncompressible.cu:20-73) or the projection alone
// (src/projectionDivergenceFree.cu:21-90), shift(+1); the tables of
// src/initializePrefactorFourierSpace.cu:39-69 evaluated in place.
template <bool ONE>
__global__ void k_inc_fourier(FSL_KARGS, int solve) {
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
    double c[3], sn[3], g[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      sincos(pi * kk[a] / (double)m[a], &sn[a], &c[a]);
      g[a] = 2 * invd[a] * sn[a];
    }
    double2 W[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double2 zz = R.z64[a * nc + i];
      W[a] = make_double2(zz.x * c[a] + zz.y * sn[a], zz.y * c[a] - zz.x * sn[a]);
    }
    double2 V[3] = {W[0], W[1], W[2]};
    if (i != 0) {
      const double GG = -(g[0] * g[0]) - (g[1] * g[1]) - (g[2] * g[2]);
      const double GWr = g[0] * W[0].x + g[1] * W[1].x + g[2] * W[2].x;
      const double GWi = g[0] * W[0].y + g[1] * W[1].y + g[2] * W[2].y;
      const double den = solve ? 1 - 0.5 * P.dt * P.eta * GG / P.rho : 1.0;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (solve)
          V[a] = make_double2((W[a].x + g[a] * GWr / GG) / den, (W[a].y + g[a] * GWi / GG) / den);
        else
          V[a] = make_double2(W[a].x + g[a] * GWr / GG, W[a].y + g[a] * GWi / GG);
      }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
      R.z64[a * nc + i] = make_double2(V[a].x * c[a] - V[a].y * sn[a], V[a].y * c[a] + V[a].x * sn[a]);
  }
}

// u^{n+1/2} = (Re(Z) / nc + u^n) / 2 into the spread buffer
// (src/realToComplex.cu:108-119)
template <bool ONE>
__global__ void k_inc_pred(FSL_KARGS) {
  FSL_REP_AT(blockIdx.y);
  const size_t n3 = 3 * (size_t)P.nc;
  double* pred = reinterpret_cast<double*>(R.grid);
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n3; k += (size_t)gridDim.x * blockDim.x)
    pred[k] = 0.5 * ((R.z64[k].x / double(P.nc)) + R.v64[k]);
}

// Z = u (src/realToComplex.cu:21-38)
template <bool ONE>
__global__ void k_inc_load(FSL_KARGS) {
  FSL_REP_AT(blockIdx.y);
  const size_t n3 = 3 * (size_t)P.nc;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n3; k += (size_t)gridDim.x * blockDim.x)
    R.z64[k] = make_double2(R.v64[k], 0.0);
}

unsigned cell_blocks(const Batch& B, long work) {
  unsigned bc = blocks_for(work, 256);
  const unsigned cap = (unsigned)((148 * 16 + B.nrep - 1) / B.nrep);
  return bc > cap ? (cap < 1 ? 1 : cap) : bc;
}

}  // namespace

void launch_inc_w(const Batch& B, int second, cudaStream_t s) {
  FSL_GO(k_inc_w, dim3(cell_blocks(B, B.nc), B.nrep), 256, 0, s, B, second);
}

void launch_inc_fourier(const Batch& B, int solve, cudaStream_t s) {
  FSL_GO(k_inc_fourier, dim3(cell_blocks(B, B.nc), B.nrep), 256, 0, s, B, solve);
}

void launch_inc_pred(const Batch& B, cudaStream_t s) {
  FSL_GO(k_inc_pred, dim3(cell_blocks(B, 3L * B.nc), B.nrep), 256, 0, s, B);
}

void launch_inc_load(const Batch& B, cudaStream_t s) {
  FSL_GO(k_inc_load, dim3(cell_blocks(B, 3L * B.nc), B.nrep), 256, 0, s, B);
}

}  // namespace fsl
