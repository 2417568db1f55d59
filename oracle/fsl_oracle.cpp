// fsl_oracle.cpp -- FP64 CPU restatement of fluam's Stokes-limit step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: the tests,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg load it to check or
// time the CUDA path.  The product (fluam_b200/) never links or calls it.
//
// It restates, in plain C++ double precision and in the same order of
// operations, the scheme of the reference (fbusabiaga/fluam):
//   src/runSchemeStokesLimit.cu:163-285            the time loop (noise, 2 solves)
//   src/boundaryParticlesFunctionStokesLimit.cu    options 0 / 1 / 2
//   src/stokesLimitFunctions.cu:23-61              non-bonded cell of a particle
//   src/stokesLimitFunctions.cu:83-1158            pair + bonded force, spread
//   src/stokesLimitFunctions.cu:1198-1681          gather (spread) with 1/dV
//   src/stokesLimitFunctions.cu:1705-2255          RFD drift spread (cell quirk)
//   src/stokesLimitFunctions.cu:2281-2378,3922-4069 W = f + c div(Sigma)
//   src/stokesLimitFunctions.cu:2399-2451          Fourier-space Stokes solve
//   src/realToComplex.cu:40-59,263-303             normalise, staggered shift
//   src/initializePrefactorFourierSpace.cu:39-69   gradK / expK tables
//   src/stokesLimitFunctions.cu:2479-2892,3513-3894 interpolation + midpoint
//   src/deltaGPU.cu:44-68                          Peskin kernels
//   src/initForcesNonBonded.cu:21-66               LJ force table (texture)
//   src/forceBondedGPU.cu:21-121                   harmonic bonds / tethers
//   src/createCellsStokesLimitGPU.cu:58-91         noise amplitudes, dx, 1/L
//   src/createBoundariesRK2GPU.cu:134-186          neighbour grid, 1/rc^2
// Third-party arithmetic that the reference takes from closed libraries is
// replaced by published algorithms: cuFFT (cufftExecZ2Z, forward sign -1,
// unnormalised) by a mixed-radix Cooley-Tukey DFT, and cuRAND's normal
// generator by the counter-based Philox4x32-10 generator (Salmon et al.,
// SC'11) with a Box-Muller transform, keyed by (seed, step, index) so that the
// CUDA path can draw the identical noise array.
//
// Extensions the reference does not have (documented in the header of
// fsl_oracle.h): soft repulsion U = eps (1 - r/rc)^2, a 3-D 4-point Peskin
// kernel, and a "paper" random-finite-difference mode that evaluates the
// drift weights at the displaced position (Delong et al., JCP 140, 134110,
// 2014, Sec. IV.B).  Compile with -ffp-contract=off: the cell index formulas
// must not be contracted into fused multiply-adds.

#include "fsl_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef std::complex<double> cplx;

// ---------------------------------------------------------------- Philox ---
struct U4 {
  uint32_t v[4];
};

inline void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
}

// Philox4x32 with 10 rounds: multipliers 0xD2511F53 / 0xCD9E8D57, Weyl key
// increments 0x9E3779B9 / 0xBB67AE85 (Salmon et al. 2011, Random123).
U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c.v[0], hi0, lo0);
    mulhilo32(0xCD9E8D57u, c.v[2], hi1, lo1);
    U4 n;
    n.v[0] = hi1 ^ c.v[1] ^ k0;
    n.v[1] = lo1;
    n.v[2] = hi0 ^ c.v[3] ^ k1;
    n.v[3] = lo0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// Normal deviate number n of draw t (one draw per time step).  Four
// consecutive indices share one Philox block; the 32-bit words are turned into
// uniforms on the open interval (0,1) with 23 random bits, u = (2 (w >> 9) + 1)
// 2^-24, which single precision represents exactly; Box-Muller pairs (u0,u1)
// and (u2,u3).
double philox_normal(uint64_t seed, uint64_t t, uint64_t n) {
  uint64_t b = n >> 2;
  U4 c;
  c.v[0] = (uint32_t)b;
  c.v[1] = (uint32_t)(b >> 32);
  c.v[2] = (uint32_t)t;
  c.v[3] = (uint32_t)(t >> 32);
  U4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  int lane = (int)(n & 3);
  int p = lane >> 1;
  double u1 = (double)(2u * (r.v[2 * p] >> 9) + 1u) * 0x1p-24;
  double u2 = (double)(2u * (r.v[2 * p + 1] >> 9) + 1u) * 0x1p-24;
  double rad = std::sqrt(-2.0 * std::log(u1));
  double ang = 2.0 * M_PI * u2;
  return (lane & 1) ? rad * std::sin(ang) : rad * std::cos(ang);
}

// ------------------------------------------------------------------- FFT ---
// Mixed-radix decimation-in-time DFT, X_k = sum_n x_n exp(sign 2 pi i k n / N),
// unnormalised (the convention of cufftExecZ2Z, sign -1 forward / +1 inverse).
struct Plan1D {
  int n = 0;
  std::vector<int> factors;
  std::vector<cplx> tw_fwd, tw_inv;  // exp(-+2 pi i t / n)
  void init(int nn) {
    n = nn;
    factors.clear();
    int m = nn;
    for (int p = 2; p * p <= m; ++p)
      while (m % p == 0) {
        factors.push_back(p);
        m /= p;
      }
    if (m > 1) factors.push_back(m);
    tw_fwd.resize(nn);
    tw_inv.resize(nn);
    for (int t = 0; t < nn; ++t) {
      double a = 2.0 * M_PI * (double)t / (double)nn;
      tw_fwd[t] = cplx(std::cos(a), -std::sin(a));
      tw_inv[t] = cplx(std::cos(a), std::sin(a));
    }
  }
};

// out[k] for the length-n sub-transform of in[0], in[s], in[2s], ...
void fft_rec(const Plan1D& P, const cplx* in, cplx* out, int n, int stride,
             int fidx, const std::vector<cplx>& tw, cplx* scratch) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  int p = P.factors[fidx];
  int m = n / p;
  // sub-transforms of the p decimated sequences, stored contiguously
  for (int r = 0; r < p; ++r)
    fft_rec(P, in + (size_t)r * stride, scratch + (size_t)r * m, m, stride * p,
            fidx + 1, tw, out);
  // combine: X[k + q m] = sum_r Y_r[k] w_n^{r (k + q m)}
  int tstep = P.n / n;  // twiddle table is for length P.n
  for (int k = 0; k < m; ++k) {
    for (int q = 0; q < p; ++q) {
      int kk = k + q * m;
      cplx acc(0.0, 0.0);
      for (int r = 0; r < p; ++r) {
        long idx = ((long)r * kk) % n;
        acc += scratch[(size_t)r * m + k] * tw[(size_t)idx * tstep];
      }
      out[kk] = acc;
    }
  }
}

void fft_line(const Plan1D& P, cplx* data, int stride, int sign,
              std::vector<cplx>& a, std::vector<cplx>& b, std::vector<cplx>& c) {
  int n = P.n;
  for (int i = 0; i < n; ++i) a[i] = data[(size_t)i * stride];
  // fft_rec needs an output buffer and a scratch buffer of length n; the
  // recursion alternates their roles, both are sized n.
  fft_rec(P, a.data(), b.data(), n, 1, 0, sign < 0 ? P.tw_fwd : P.tw_inv,
          c.data());
  for (int i = 0; i < n; ++i) data[(size_t)i * stride] = b[i];
}

// 3-D transform of one component stored x-fastest, index x + y mx + z mx my
// (the cufftPlan3d(mz, my, mx) layout of src/runSchemeStokesLimit.cu:135).
void fft3d(cplx* d, int mx, int my, int mz, const Plan1D& Px, const Plan1D& Py,
           const Plan1D& Pz, int sign) {
  int mmax = std::max(mx, std::max(my, mz));
#pragma omp parallel
  {
    std::vector<cplx> a(mmax), b(mmax), c(mmax);
#pragma omp for collapse(2) schedule(static)
    for (int z = 0; z < mz; ++z)
      for (int y = 0; y < my; ++y)
        fft_line(Px, d + (size_t)mx * (y + (size_t)my * z), 1, sign, a, b, c);
#pragma omp for collapse(2) schedule(static)
    for (int z = 0; z < mz; ++z)
      for (int x = 0; x < mx; ++x)
        fft_line(Py, d + x + (size_t)mx * my * z, mx, sign, a, b, c);
#pragma omp for collapse(2) schedule(static)
    for (int y = 0; y < my; ++y)
      for (int x = 0; x < mx; ++x)
        fft_line(Pz, d + x + (size_t)mx * y, mx * my, sign, a, b, c);
  }
}

// ------------------------------------------------------- small helpers -----
inline double sgn(double r) { return (double)((r > 0) - (r < 0)); }

// Minimum image r - int(r/L + sign(r)/2) L (src/stokesLimitFunctions.cu:41-49).
inline double minimage(double r, double invL, double L) {
  return r - (double)(int)(r * invL + 0.5 * sgn(r)) * L;
}

// Cell index int(r m/L + m/2) % m of an already wrapped coordinate.
inline int cellidx(double r, double invd, int m) {
  return (int)(r * invd + 0.5 * (double)m) % m;
}

// 3-point Peskin kernel of src/deltaGPU.cu:57-68, including its sqrtf.
inline double delta3(double x) {
  x = std::fabs(x);
  if (x > 1.5) return 0.0;
  if (x < 0.5) return (1. + (double)sqrtf((float)(1. - 3. * x * x))) / 3.;
  return (5. - 3. * x - (double)sqrtf((float)(1. - 3. * (1. - x) * (1. - x)))) / 6.;
}

// 4-point Peskin kernel (Peskin, Acta Numerica 2002, eq. 6.27), the 3-D
// extension; the reference only has the fractional-offset form of it
// (src/deltaGPU.cu:44-53).
inline double delta4(double x) {
  x = std::fabs(x);
  if (x >= 2.0) return 0.0;
  if (x <= 1.0) return (3. - 2. * x + std::sqrt(1. + 4. * x - 4. * x * x)) / 8.;
  return (5. - 2. * x - std::sqrt(-7. + 12. * x - 4. * x * x)) / 8.;
}

// Linear filtering of a normalised, clamped 1-D float texture: the CUDA
// texture unit uses x_B = x N - 1/2, i = floor(x_B), and a fractional weight
// held in 9-bit fixed point with 8 fractional bits.  The weight is rounded to
// the nearest 1/256 here; the CUDA path uses the same formula in software.
inline float tex_linear(const float* T, int N, float x) {
  double xb = (double)x * (double)N - 0.5;
  double fl = std::floor(xb);
  int i = (int)fl;
  float a = (float)(std::nearbyint((xb - fl) * 256.0) / 256.0);
  int i0 = std::min(std::max(i, 0), N - 1);
  int i1 = std::min(std::max(i + 1, 0), N - 1);
  return (1.0f - a) * T[i0] + a * T[i1];
}

}  // namespace

// ------------------------------------------------------------- the state ---
struct orc_state {
  orc_config c;
  // grid
  int mx, my, mz, nc;
  double dx, dy, dz, invdx, invdy, invdz, invlx, invly, invlz, dV;
  double fact1, fact2, fact4;
  Plan1D Px, Py, Pz;
  std::vector<double> gradK[3], expKre[3], expKim[3];
  // neighbour grid (non-bonded)
  int mnx, mny, mnz, mN;
  double invcut2;
  std::vector<float> ljtab;
  // particles
  int np;
  std::vector<double> q, qp, F;  // SoA x|y|z
  // bonds (CSR, both endpoints store each bond)
  bool bonded = false;
  std::vector<int> bpp_cnt, bpp_off, bpp_idx;
  std::vector<double> bpp_k, bpp_r0;
  std::vector<int> bfp_cnt, bfp_off;
  std::vector<double> bfp_k, bfp_r0, bfp_xyz;
  // fields
  std::vector<double> f, v, acc;
  std::vector<cplx> Z;
  std::vector<double> noise;
  // non-bonded cell list (ascending particle index inside a cell)
  std::vector<int> cell_of, cstart, csorted;
  // quasi-2D family (src/createCellsQuasi2DGPU.cu:49-98): Gaussian variance,
  // stencil half-width, stochastic prefactor
  double q2_var = 0.0, q2_fact1 = 0.0;
  int q2_kw = 0;
  uint64_t t = 0;
};

namespace {

void build_ljtable(orc_state* s) {
  // src/initForcesNonBonded.cu:21-53: float accumulation of r, float sqrt,
  // sigma = 2 dx and epsilon = kT hard-coded, entries 0 and 4095 zeroed.
  const int size = 4096;
  s->ljtab.assign(size, 0.0f);
  float sigma = (float)(2.0 * s->c.lx / (double)s->mx);
  float epsilon = (float)s->c.temperature;
  float cutoff2 = (float)(s->c.cutoff * s->c.cutoff);
  float dr = cutoff2 / (float)size;
  float r = 0.5f * dr;
  for (int i = 0; i < size; ++i) {
    double rr = (double)sqrtf(r);
    float fr = (float)(48. * epsilon *
                       (std::pow(sigma / rr, 12) - 0.5 * std::pow(sigma / rr, 6)) / rr);
    s->ljtab[i] = fr / sqrtf(r);
    r += dr;
  }
  s->ljtab[size - 1] = 0.0f;
  s->ljtab[0] = 0.0f;
}

// Non-bonded cell of a coordinate triple (src/stokesLimitFunctions.cu:31-46).
inline int nb_cell(const orc_state* s, double rx, double ry, double rz) {
  double invdx = (double)s->mnx / s->c.lx;
  double invdy = (double)s->mny / s->c.ly;
  double invdz = (double)s->mnz / s->c.lz;
  rx = minimage(rx, s->invlx, s->c.lx);
  int jx = cellidx(rx, invdx, s->mnx);
  ry = minimage(ry, s->invly, s->c.ly);
  int jy = cellidx(ry, invdy, s->mny);
  rz = minimage(rz, s->invlz, s->c.lz);
  int jz = cellidx(rz, invdz, s->mnz);
  return jx + jy * s->mnx + jz * s->mnx * s->mny;
}

void build_cells(orc_state* s, const double* q) {
  int np = s->np;
  s->cell_of.assign(np, 0);
  std::vector<int> cnt(s->mN + 1, 0);
  for (int i = 0; i < np; ++i) {
    int c = nb_cell(s, q[i], q[np + i], q[2 * np + i]);
    s->cell_of[i] = c;
    cnt[c + 1]++;
  }
  s->cstart.assign(s->mN + 1, 0);
  for (int c = 0; c < s->mN; ++c) s->cstart[c + 1] = s->cstart[c] + cnt[c + 1];
  std::vector<int> fill(s->cstart.begin(), s->cstart.end() - 1);
  s->csorted.assign(np, 0);
  for (int i = 0; i < np; ++i) s->csorted[fill[s->cell_of[i]]++] = i;
}

// Neighbour-cell order of the pair loop, src/stokesLimitFunctions.cu:191-653:
// own cell, -z, -y, -x, +x, +y, +z, then the 12 edge and 8 corner cells.
const int kNbOrder[27][3] = {
    {0, 0, 0},   {0, 0, -1},  {0, -1, 0},  {-1, 0, 0},  {1, 0, 0},   {0, 1, 0},
    {0, 0, 1},   {1, 1, 0},   {1, -1, 0},  {1, 0, 1},   {1, 0, -1},  {-1, 1, 0},
    {-1, -1, 0}, {-1, 0, 1},  {-1, 0, -1}, {0, 1, 1},   {0, 1, -1},  {0, -1, 1},
    {0, -1, -1}, {1, 1, 1},   {1, 1, -1},  {1, -1, 1},  {1, -1, -1}, {-1, 1, 1},
    {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};

// Force on every particle at positions q (cell list must be built for q).
void compute_forces(orc_state* s, const double* q, double* F) {
  int np = s->np;
  const double lx = s->c.lx, ly = s->c.ly, lz = s->c.lz;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < np; ++i) {
    double fx = 0., fy = 0., fz = 0.;
    double rx = q[i], ry = q[np + i], rz = q[2 * np + i];
    if (s->bonded) {
      // src/forceBondedGPU.cu:37-113, no minimum image on bonds
      int nb = s->bpp_cnt[i], off = s->bpp_off[i];
      for (int j = 0; j < nb; ++j) {
        int idx = s->bpp_idx[off + j];
        double x = q[idx], y = q[np + idx], z = q[2 * np + idx];
        double r0 = s->bpp_r0[off + j], k = s->bpp_k[off + j];
        if (r0 == 0) {
          fx += -k * (rx - x);
          fy += -k * (ry - y);
          fz += -k * (rz - z);
        } else {
          double r = std::sqrt((x - rx) * (x - rx) + (y - ry) * (y - ry) + (z - rz) * (z - rz));
          if (r > 0) {
            fx += -k * (1 - r0 / r) * (rx - x);
            fy += -k * (1 - r0 / r) * (ry - y);
            fz += -k * (1 - r0 / r) * (rz - z);
          }
        }
      }
      nb = s->bfp_cnt[i];
      off = s->bfp_off[i];
      for (int j = 0; j < nb; ++j) {
        double x = s->bfp_xyz[3 * (off + j)], y = s->bfp_xyz[3 * (off + j) + 1],
               z = s->bfp_xyz[3 * (off + j) + 2];
        double r0 = s->bfp_r0[off + j], k = s->bfp_k[off + j];
        if (r0 == 0) {
          fx += -k * (rx - x);
          fy += -k * (ry - y);
          fz += -k * (rz - z);
        } else {
          double r = std::sqrt((x - rx) * (x - rx) + (y - ry) * (y - ry) + (z - rz) * (z - rz));
          if (r > 0) {
            fx += -k * (1 - r0 / r) * (rx - x);
            fy += -k * (1 - r0 / r) * (ry - y);
            fz += -k * (1 - r0 / r) * (rz - z);
          }
        }
      }
    }
    if (s->c.nonbonded && s->c.pair != ORC_PAIR_NONE) {
      int c = s->cell_of[i];
      int cx = c % s->mnx, cy = (c / s->mnx) % s->mny, cz = c / (s->mnx * s->mny);
      for (int nn = 0; nn < 27; ++nn) {
        int ox = (cx + kNbOrder[nn][0] + s->mnx) % s->mnx;
        int oy = (cy + kNbOrder[nn][1] + s->mny) % s->mny;
        int oz = (cz + kNbOrder[nn][2] + s->mnz) % s->mnz;
        int cc = ox + oy * s->mnx + oz * s->mnx * s->mny;
        for (int jj = s->cstart[cc]; jj < s->cstart[cc + 1]; ++jj) {
          int j = s->csorted[jj];
          double rxij = rx - q[j];
          rxij = rxij - (double)(int)(rxij * s->invlx + 0.5 * sgn(rxij)) * lx;
          double ryij = ry - q[np + j];
          ryij = ryij - (double)(int)(ryij * s->invly + 0.5 * sgn(ryij)) * ly;
          double rzij = rz - q[2 * np + j];
          rzij = rzij - (double)(int)(rzij * s->invlz + 0.5 * sgn(rzij)) * lz;
          double r2 = rxij * rxij + ryij * ryij + rzij * rzij;
          double f = 0.0;
          if (s->c.pair == ORC_PAIR_TABLE_LJ) {
            f = (double)tex_linear(s->ljtab.data(), 4096, (float)(r2 * s->invcut2));
          } else {  // soft repulsion, F(r)/r = (2 eps / rc)(1 - r/rc)/r, r < rc
            if (j == i || r2 >= s->c.cutoff * s->c.cutoff || r2 == 0.0) continue;
            double r = std::sqrt(r2);
            f = (2.0 * s->c.soft_epsilon / s->c.cutoff) * (1.0 - r / s->c.cutoff) / r;
          }
          fx += f * rxij;
          fy += f * ryij;
          fz += f * rzij;
        }
      }
    }
    F[i] = fx;
    F[np + i] = fy;
    F[2 * np + i] = fz;
  }
}

// Stencil of one particle for field component `comp` (0 x-faces, 1 y-faces,
// 2 z-faces): for each dimension the first node index and the weights.
struct Stencil {
  int n;          // 3 or 4 nodes per dimension
  int j0[3];      // first node index (periodic, 0..m-1)
  double w[3][4];
};

// Nodes of component comp in dimension d sit at (j + 1/2) h - L/2, shifted by
// +h/2 when d == comp (the face of cell j).  posw is the position that sets
// the weights, posc the one that picks the nodes (they differ only in the
// RFD cell quirk, src/stokesLimitFunctions.cu:1749-1803 vs 1872-1918).
void stencil(const orc_state* s, int comp, const double posc[3], const double posw[3],
             Stencil& st) {
  const int m[3] = {s->mx, s->my, s->mz};
  const double h[3] = {s->dx, s->dy, s->dz};
  const double invd[3] = {s->invdx, s->invdy, s->invdz};
  const double L[3] = {s->c.lx, s->c.ly, s->c.lz};
  const double invL[3] = {s->invlx, s->invly, s->invlz};
  st.n = s->c.kernel == 4 ? 4 : 3;
  for (int d = 0; d < 3; ++d) {
    double off = (d == comp) ? 0.5 * h[d] : 0.0;
    if (st.n == 3) {
      // nearest node (src/stokesLimitFunctions.cu:662-698)
      double r = posc[d] - off;
      r = minimage(r, invL[d], L[d]);
      int jc = cellidx(r, invd[d], m[d]);
      st.j0[d] = (jc - 1 + m[d]) % m[d];
      double aux = invd[d] / 1.5;
      for (int k = 0; k < 3; ++k) {
        int j = (st.j0[d] + k) % m[d];
        double node = ((double)j + 0.5) * h[d] - 0.5 * L[d];  // cell centre
        double rr = posw[d] - node - off;
        rr = aux * (rr - (double)(int)(rr * invL[d] + 0.5 * sgn(rr)) * L[d]);
        st.w[d][k] = delta3(1.5 * rr);
      }
      st.w[d][3] = 0.0;
    } else {
      // node at or below the position, then one below and two above
      double r = posc[d] - off - 0.5 * h[d];
      r = minimage(r, invL[d], L[d]);
      int jb = cellidx(r, invd[d], m[d]);
      st.j0[d] = (jb - 1 + m[d]) % m[d];
      for (int k = 0; k < 4; ++k) {
        int j = (st.j0[d] + k) % m[d];
        double node = ((double)j + 0.5) * h[d] - 0.5 * L[d] + off;
        double rr = minimage(posw[d] - node, invL[d], L[d]) * invd[d];
        st.w[d][k] = delta4(rr);
      }
    }
  }
}

// acc[comp][node] += w * value for every particle, in particle order.
void spread_values(orc_state* s, const double* qc, const double* qw, const double* val,
                   double* accg) {
  int np = s->np, nc = s->nc;
  const int mx = s->mx, my = s->my, mz = s->mz;
#pragma omp parallel for schedule(static, 1)
  for (int comp = 0; comp < 3; ++comp) {
    double* a = accg + (size_t)comp * nc;
    for (int i = 0; i < np; ++i) {
      double pc[3] = {qc[i], qc[np + i], qc[2 * np + i]};
      double pw[3] = {qw[i], qw[np + i], qw[2 * np + i]};
      Stencil st;
      stencil(s, comp, pc, pw, st);
      double F = val[(size_t)comp * np + i];
      for (int a0 = 0; a0 < st.n; ++a0) {
        int x = (st.j0[0] + a0) % mx;
        for (int b0 = 0; b0 < st.n; ++b0) {
          int y = (st.j0[1] + b0) % my;
          double wxy = st.w[0][a0] * st.w[1][b0];
          for (int c0 = 0; c0 < st.n; ++c0) {
            int z = (st.j0[2] + c0) % mz;
            a[x + (size_t)mx * (y + (size_t)my * z)] += wxy * st.w[2][c0] * F;
          }
        }
      }
    }
  }
}

// f += S(q) val / dV  (one spread kernel + one gather pass of the reference)
void spread_add(orc_state* s, const double* qc, const double* qw, const double* val) {
  std::fill(s->acc.begin(), s->acc.end(), 0.0);
  spread_values(s, qc, qw, val, s->acc.data());
  size_t n3 = (size_t)3 * s->nc;
#pragma omp parallel for schedule(static)
  for (size_t k = 0; k < n3; ++k) s->f[k] += s->acc[k] / s->dV;
}

// u = J(q) v : interpolation with the same stencils, no volume factor.
void interpolate(const orc_state* s, const double* q, const double* v, double* u) {
  int np = s->np, nc = s->nc;
  const int mx = s->mx, my = s->my, mz = s->mz;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < np; ++i) {
    double p[3] = {q[i], q[np + i], q[2 * np + i]};
    for (int comp = 0; comp < 3; ++comp) {
      Stencil st;
      stencil(s, comp, p, p, st);
      const double* vc = v + (size_t)comp * nc;
      double sum = 0.0;
      for (int a0 = 0; a0 < st.n; ++a0) {
        int x = (st.j0[0] + a0) % mx;
        for (int b0 = 0; b0 < st.n; ++b0) {
          int y = (st.j0[1] + b0) % my;
          for (int c0 = 0; c0 < st.n; ++c0) {
            int z = (st.j0[2] + c0) % mz;
            sum += st.w[0][a0] * st.w[1][b0] * st.w[2][c0] *
                   vc[x + (size_t)mx * (y + (size_t)my * z)];
          }
        }
      }
      u[(size_t)comp * np + i] = sum;
    }
  }
}

// W = f + noiseFactor div(Sigma) (src/stokesLimitFunctions.cu:2281-2378 and,
// with two stress samples, 3922-4069).  W is written as the real part of Z.
void construct_W(orc_state* s, double noiseFactor, bool second) {
  const int mx = s->mx, my = s->my, mz = s->mz, nc = s->nc;
  const double* R = s->noise.data();
  const size_t off2 = (size_t)6 * nc + (size_t)9 * s->np;
  const double fact1 = noiseFactor * s->fact1, fact4 = noiseFactor * s->fact4;
  const double invdx = s->invdx, invdy = s->invdy, invdz = s->invdz;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nc; ++i) {
    int x = i % mx, y = (i / mx) % my, z = i / (mx * my);
    int v0 = x + mx * (y + my * ((z - 1 + mz) % mz));  // -z
    int v1 = x + mx * (((y - 1 + my) % my) + my * z);  // -y
    int v2 = (x - 1 + mx) % mx + mx * (y + my * z);    // -x
    int v3 = (x + 1) % mx + mx * (y + my * z);         // +x
    int v4 = x + mx * (((y + 1) % my) + my * z);       // +y
    int v5 = x + mx * (y + my * ((z + 1) % mz));       // +z
    double wx = s->f[i], wy = s->f[nc + i], wz = s->f[2 * nc + i];
    int nsets = second ? 2 : 1;
    for (int set = 0; set < nsets; ++set) {
      const double* d = R + (set ? off2 : 0);
      double n;
      n = d[v3];                       wx += invdx * fact1 * n;
      n = d[v4 + 3 * nc];              wy += invdy * fact1 * n;
      n = d[v5 + 5 * nc];              wz += invdz * fact1 * n;
      n = d[i + nc];                   wx += invdy * fact4 * n; wy += invdx * fact4 * n;
      n = d[i + 2 * nc];               wx += invdz * fact4 * n; wz += invdx * fact4 * n;
      n = d[i + 4 * nc];               wy += invdz * fact4 * n; wz += invdy * fact4 * n;
      n = d[i];                        wx -= invdx * fact1 * n;
      n = d[i + 3 * nc];               wy -= invdy * fact1 * n;
      n = d[i + 5 * nc];               wz -= invdz * fact1 * n;
      n = d[v1 + nc];                  wx -= invdy * fact4 * n;
      n = d[v0 + 2 * nc];              wx -= invdz * fact4 * n;
      n = d[v2 + nc];                  wy -= invdx * fact4 * n;
      n = d[v0 + 4 * nc];              wy -= invdz * fact4 * n;
      n = d[v2 + 2 * nc];              wz -= invdx * fact4 * n;
      n = d[v1 + 4 * nc];              wz -= invdy * fact4 * n;
    }
    s->Z[i] = cplx(wx, 0.0);
    s->Z[nc + i] = cplx(wy, 0.0);
    s->Z[2 * nc + i] = cplx(wz, 0.0);
  }
}

// v = (eta L)^-1 P W : forward FFT, shift(-1), projection / divide,
// shift(+1), inverse FFT, Re / ncells.
void solve(orc_state* s) {
  const int mx = s->mx, my = s->my, mz = s->mz, nc = s->nc;
  for (int comp = 0; comp < 3; ++comp)
    fft3d(s->Z.data() + (size_t)comp * nc, mx, my, mz, s->Px, s->Py, s->Pz, -1);
  const double eta = s->c.shearviscosity;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nc; ++i) {
    int kz = i / (mx * my), ky = (i % (mx * my)) / mx, kx = i % mx;
    cplx W[3] = {s->Z[i], s->Z[nc + i], s->Z[2 * nc + i]};
    const int kk[3] = {kx, ky, kz};
    // kernelShift(-1): W_a * (cos - i sin) (src/realToComplex.cu:263-303)
    for (int a = 0; a < 3; ++a) {
      double c = s->expKre[a][kk[a]], sn = s->expKim[a][kk[a]];
      double re = W[a].real() * c - (-1) * W[a].imag() * sn;
      double im = W[a].imag() * c + (-1) * W[a].real() * sn;
      W[a] = cplx(re, im);
    }
    double gx = s->gradK[0][kx], gy = s->gradK[1][ky], gz = s->gradK[2][kz];
    double L = -(gx * gx) - (gy * gy) - (gz * gz);
    double GG = L;
    double denominator = -eta * L;
    double GWr = gx * W[0].real() + gy * W[1].real() + gz * W[2].real();
    double GWi = gx * W[0].imag() + gy * W[1].imag() + gz * W[2].imag();
    cplx V[3];
    if (i == 0) {
      V[0] = V[1] = V[2] = cplx(0.0, 0.0);
    } else {
      const double g[3] = {gx, gy, gz};
      for (int a = 0; a < 3; ++a)
        V[a] = cplx((W[a].real() + g[a] * GWr / GG) / denominator,
                    (W[a].imag() + g[a] * GWi / GG) / denominator);
    }
    // kernelShift(+1)
    for (int a = 0; a < 3; ++a) {
      double c = s->expKre[a][kk[a]], sn = s->expKim[a][kk[a]];
      double re = V[a].real() * c - (1) * V[a].imag() * sn;
      double im = V[a].imag() * c + (1) * V[a].real() * sn;
      s->Z[(size_t)a * nc + i] = cplx(re, im);
    }
  }
  for (int comp = 0; comp < 3; ++comp)
    fft3d(s->Z.data() + (size_t)comp * nc, mx, my, mz, s->Px, s->Py, s->Pz, +1);
  size_t n3 = (size_t)3 * nc;
#pragma omp parallel for schedule(static)
  for (size_t k = 0; k < n3; ++k) s->v[k] = s->Z[k].real() / (double)nc;
}

void draw_noise(orc_state* s) {
  size_t n = (size_t)12 * s->nc + (size_t)9 * s->np;
  s->noise.resize(n);
  uint64_t seed = s->c.seed, t = s->t;
#pragma omp parallel for schedule(static)
  for (size_t k = 0; k < n; ++k) s->noise[k] = philox_normal(seed, t, k);
}

// RFD drift forces for one sign: (kT/delta) sign W_p, spread from the
// displaced position q + sign (delta/2) W_p (nodes) with weights taken at q
// (reference mode) or at the displaced position (paper mode).
void spread_drift(orc_state* s, int sign) {
  int np = s->np, nc = s->nc;
  const double delta = 0.001;
  const double fpre = (s->c.temperature / delta) * sign;
  std::vector<double> val(3 * (size_t)np), qd(3 * (size_t)np);
  for (int d = 0; d < 3; ++d)
    for (int i = 0; i < np; ++i) {
      double W = s->noise[(size_t)6 * nc + (size_t)d * np + i];
      val[(size_t)d * np + i] = fpre * W;
      qd[(size_t)d * np + i] = s->q[(size_t)d * np + i] + sign * 0.5 * delta * W;
    }
  if (s->c.rfd == ORC_RFD_PAPER)
    spread_add(s, qd.data(), qd.data(), val.data());
  else
    spread_add(s, qd.data(), s->q.data(), val.data());
}

// One step of the first-order scheme, src/runSchemeStokesLimitFirstOrder.cu
// :163-241 with src/boundaryParticlesFunctionStokesLimitFirstOrder.cu:32-214:
// one solve with f = S(q^n) F^n + RFD drift and noise factor 1, then the
// predictor and corrector of the midpoint step with the same velocity field;
// forces at q^{n+1/2} only with extraMobility (particlesForceStokesLimit).
void one_step_first_order(orc_state* s) {
  const int np = s->np, nc = s->nc;
  const double dt = s->c.dt;
  draw_noise(s);
  std::vector<double> u(3 * (size_t)np);
  std::fill(s->f.begin(), s->f.end(), 0.0);
  if (np > 0) {
    build_cells(s, s->q.data());
    compute_forces(s, s->q.data(), s->F.data());
    spread_add(s, s->q.data(), s->q.data(), s->F.data());
    spread_drift(s, +1);
    spread_drift(s, -1);
  }
  construct_W(s, 1.0, false);
  solve(s);
  if (np > 0) {
    interpolate(s, s->q.data(), s->v.data(), u.data());
    for (int d = 0; d < 3; ++d)
      for (int i = 0; i < np; ++i) {
        size_t k = (size_t)d * np + i;
        double rnew = s->q[k] + 0.5 * dt * u[k];
        if (s->c.extra_mobility != 0.0)
          rnew += 0.5 * dt * s->c.extra_mobility * s->F[k] +
                  s->fact2 * s->noise[(size_t)6 * nc + (size_t)(3 + d) * np + i];
        s->qp[k] = rnew;
      }
    if (s->c.extra_mobility != 0.0) {
      build_cells(s, s->qp.data());
      compute_forces(s, s->qp.data(), s->F.data());
    }
    interpolate(s, s->qp.data(), s->v.data(), u.data());
    for (int d = 0; d < 3; ++d)
      for (int i = 0; i < np; ++i) {
        size_t k = (size_t)d * np + i;
        double rnew = s->q[k] + dt * u[k];
        if (s->c.extra_mobility != 0.0)
          rnew += dt * s->c.extra_mobility * s->F[k] +
                  s->fact2 * (s->noise[(size_t)6 * nc + (size_t)(3 + d) * np + i] +
                              s->noise[(size_t)6 * nc + (size_t)(6 + d) * np + i]);
        s->q[k] = rnew;
      }
  }
  s->t++;
}

void one_step_q2d(orc_state* s);
void one_step_incompressible(orc_state* s);

void one_step(orc_state* s) {
  if (s->c.scheme == ORC_SCHEME_FIRST_ORDER) return one_step_first_order(s);
  if (s->c.scheme == ORC_SCHEME_QUASI2D || s->c.scheme == ORC_SCHEME_STOKES2D) return one_step_q2d(s);
  if (s->c.scheme == ORC_SCHEME_INCOMPRESSIBLE) return one_step_incompressible(s);
  const int np = s->np, nc = s->nc;
  const double dt = s->c.dt;
  draw_noise(s);
  std::vector<double> u(3 * (size_t)np);
  // ---- option 0: forces at q^n, f = S F
  std::fill(s->f.begin(), s->f.end(), 0.0);
  if (np > 0) {
    build_cells(s, s->q.data());
    compute_forces(s, s->q.data(), s->F.data());
    spread_add(s, s->q.data(), s->q.data(), s->F.data());
  }
  construct_W(s, std::sqrt(2.0), false);
  solve(s);
  // ---- option 1: predictor, forces at q^{n+1/2}, RFD
  if (np > 0) {
    interpolate(s, s->q.data(), s->v.data(), u.data());
    for (int d = 0; d < 3; ++d)
      for (int i = 0; i < np; ++i) {
        size_t k = (size_t)d * np + i;
        double rnew = s->q[k] + 0.5 * dt * u[k];
        if (s->c.extra_mobility != 0.0)
          rnew += 0.5 * dt * s->c.extra_mobility * s->F[k] +
                  s->fact2 * s->noise[(size_t)6 * nc + (size_t)(3 + d) * np + i];
        s->qp[k] = rnew;
      }
  }
  std::fill(s->f.begin(), s->f.end(), 0.0);
  if (np > 0) {
    build_cells(s, s->qp.data());
    compute_forces(s, s->qp.data(), s->F.data());
    spread_add(s, s->qp.data(), s->qp.data(), s->F.data());
    spread_drift(s, +1);
    spread_drift(s, -1);
  }
  construct_W(s, std::sqrt(0.5), true);
  solve(s);
  // ---- option 2: corrector
  if (np > 0) {
    interpolate(s, s->qp.data(), s->v.data(), u.data());
    for (int d = 0; d < 3; ++d)
      for (int i = 0; i < np; ++i) {
        size_t k = (size_t)d * np + i;
        double rnew = s->q[k] + dt * u[k];
        if (s->c.extra_mobility != 0.0)
          rnew += dt * s->c.extra_mobility * s->F[k] +
                  s->fact2 * (s->noise[(size_t)6 * nc + (size_t)(3 + d) * np + i] +
                              s->noise[(size_t)6 * nc + (size_t)(6 + d) * np + i]);
        s->q[k] = rnew;
      }
  }
  s->t++;
}

// ========================================= incompressible fluid (3D) ===
// The fluctuating incompressible Navier-Stokes solver of keyword
// incompressible (src/runSchemeIncompressible.cu:20-155): staggered
// velocities, Crank-Nicolson viscous term and a midpoint advection in two
// substeps sharing one noise draw, the projection done in Fourier space.

// W = u + dt/2 (eta/rho) L u - (dt/4) A(a) + div(Sigma) per cell, the
// advection A taken from field a (u in the first substep, the prediction in
// the second), src/kernelConstructW.cu:32-265 and 266-521; written as the
// real part of Z.
void inc_build_W(orc_state* s, const double* a) {
  const int mx = s->mx, my = s->my, mz = s->mz, nc = s->nc;
  const double* u = s->v.data();
  const double* R = s->noise.data();
  const double idx = s->invdx, idy = s->invdy, idz = s->invdz, dt = s->c.dt;
  const double nu = s->c.shearviscosity / s->c.density;
  const double f1 = s->fact1, f4 = s->fact4;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nc; ++i) {
    const int x = i % mx, y = (i / mx) % my, z = i / (mx * my);
    auto at = [&](int dx, int dy, int dz) {
      return (x + dx + mx) % mx + mx * (((y + dy + my) % my) + my * ((z + dz + mz) % mz));
    };
    const int v0 = at(0, 0, -1), v1 = at(0, -1, 0), v2 = at(-1, 0, 0), v3 = at(1, 0, 0),
              v4 = at(0, 1, 0), v5 = at(0, 0, 1);
    const int pxmy = at(1, -1, 0), pxmz = at(1, 0, -1), mxpy = at(-1, 1, 0), mxpz = at(-1, 0, 1),
              pymz = at(0, 1, -1), mypz = at(0, -1, 1);
    const double* ux = u;
    const double* uy = u + nc;
    const double* uz = u + 2 * (size_t)nc;
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
    // advection of a (momentum flux differences at the faces)
    const double* ax = a;
    const double* ay = a + nc;
    const double* az = a + 2 * (size_t)nc;
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
    // divergence of the traceless symmetric random stress, layout
    // XX, XY, XZ, YY, YZ, ZZ (src/kernelConstructW.cu:158-212)
    const size_t n = nc;
    auto trace = [&](int c) { return R[c] + R[c + 3 * n] + R[c + 5 * n]; };
    wx += idx * f1 * (R[v3] - trace(v3) / 3.);
    wy += idy * f1 * (R[v4 + 3 * n] - trace(v4) / 3.);
    wz += idz * f1 * (R[v5 + 5 * n] - trace(v5) / 3.);
    wx += idy * f4 * R[i + n];
    wy += idx * f4 * R[i + n];
    wx += idz * f4 * R[i + 2 * n];
    wz += idx * f4 * R[i + 2 * n];
    wy += idz * f4 * R[i + 4 * n];
    wz += idy * f4 * R[i + 4 * n];
    const double tr = trace(i);
    wx -= idx * f1 * (R[i] - tr / 3.);
    wy -= idy * f1 * (R[i + 3 * n] - tr / 3.);
    wz -= idz * f1 * (R[i + 5 * n] - tr / 3.);
    wx -= idy * f4 * R[v1 + n];
    wx -= idz * f4 * R[v0 + 2 * n];
    wy -= idx * f4 * R[v2 + n];
    wy -= idz * f4 * R[v0 + 4 * n];
    wz -= idx * f4 * R[v2 + 2 * n];
    wz -= idy * f4 * R[v1 + 4 * n];
    s->Z[i] = cplx(wx, 0.0);
    s->Z[nc + i] = cplx(wy, 0.0);
    s->Z[2 * nc + i] = cplx(wz, 0.0);
  }
}

// Per mode of Z: shift(-1), then either the Crank-Nicolson solve
// (src/kernelUpdateVIncompressible.cu:20-73) or the projection alone
// (src/projectionDivergenceFree.cu:21-90), then shift(+1).
void inc_fourier(orc_state* s, bool solve) {
  const int mx = s->mx, my = s->my, nc = s->nc;
  const double dt = s->c.dt, eta = s->c.shearviscosity, rho = s->c.density;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nc; ++i) {
    const int kz = i / (mx * my), ky = (i % (mx * my)) / mx, kx = i % mx;
    const int kk[3] = {kx, ky, kz};
    cplx W[3] = {s->Z[i], s->Z[nc + i], s->Z[2 * (size_t)nc + i]};
    for (int a = 0; a < 3; ++a) {
      const double c = s->expKre[a][kk[a]], sn = s->expKim[a][kk[a]];
      W[a] = cplx(W[a].real() * c + W[a].imag() * sn, W[a].imag() * c - W[a].real() * sn);
    }
    const double g[3] = {s->gradK[0][kx], s->gradK[1][ky], s->gradK[2][kz]};
    const double GG = -(g[0] * g[0]) - (g[1] * g[1]) - (g[2] * g[2]);
    const double GWr = g[0] * W[0].real() + g[1] * W[1].real() + g[2] * W[2].real();
    const double GWi = g[0] * W[0].imag() + g[1] * W[1].imag() + g[2] * W[2].imag();
    cplx V[3] = {W[0], W[1], W[2]};
    if (i != 0) {
      const double den = solve ? 1 - 0.5 * dt * eta * GG / rho : 1.0;
      for (int a = 0; a < 3; ++a) {
        if (solve)
          V[a] = cplx((W[a].real() + g[a] * GWr / GG) / den, (W[a].imag() + g[a] * GWi / GG) / den);
        else
          V[a] = cplx(W[a].real() + g[a] * GWr / GG, W[a].imag() + g[a] * GWi / GG);
      }
    }
    for (int a = 0; a < 3; ++a) {
      const double c = s->expKre[a][kk[a]], sn = s->expKim[a][kk[a]];
      s->Z[(size_t)a * nc + i] = cplx(V[a].real() * c - V[a].imag() * sn, V[a].imag() * c + V[a].real() * sn);
    }
  }
}

void inc_transform(orc_state* s, int sign) {
  for (int comp = 0; comp < 3; ++comp)
    fft3d(s->Z.data() + (size_t)comp * s->nc, s->mx, s->my, s->mz, s->Px, s->Py, s->Pz, sign);
}

// One step of runSchemeIncompressible (src/runSchemeIncompressible.cu:98-146).
void one_step_incompressible(orc_state* s) {
  const int nc = s->nc;
  const size_t n3 = 3 * (size_t)nc;
  {
    const size_t n = (size_t)6 * nc;
    s->noise.resize(n);
    for (size_t k = 0; k < n; ++k) s->noise[k] = philox_normal(s->c.seed, s->t, k);
  }
  inc_build_W(s, s->v.data());
  inc_transform(s, -1);
  inc_fourier(s, true);
  inc_transform(s, +1);
  // prediction u^{n+1/2} = (u^n + u*) / 2 (src/realToComplex.cu:108-119)
  std::vector<double> pred(n3);
  for (size_t k = 0; k < n3; ++k) pred[k] = 0.5 * ((s->Z[k].real() / double(nc)) + s->v[k]);
  inc_build_W(s, pred.data());
  inc_transform(s, -1);
  inc_fourier(s, true);
  inc_transform(s, +1);
  for (size_t k = 0; k < n3; ++k) s->v[k] = s->Z[k].real() / (double)nc;
  s->t++;
}

// ================================================ quasi-2D family (2D) ===
// The Gaussian-blob Stokes schemes of keywords quasi2D (RPY mobility of a
// blob in a quasi-2D geometry) and stokesLimit2D (2-D Stokes, optionally
// Saffman-screened), src/runSchemeQuasi2D.cu:20-260.  Grid nodes sit at the
// cell corners x_k = k dx - lx/2; a particle's stencil is the (2w+1)^2 nodes
// around the node at or below it (w = kernelWidth).  Fields are complex
// [2][my][mx] (x fastest), FP64 throughout as in the reference.

inline bool q2_scheme(const orc_state* s) {
  return s->c.scheme == ORC_SCHEME_QUASI2D || s->c.scheme == ORC_SCHEME_STOKES2D;
}

// src/deltaGPU.cu:114-117
inline double gauss2d(double r2, double var) {
  const double pi = 3.1415926535897932385;
  return std::exp(-r2 / (2.0 * var)) / (2 * pi * var);
}

// (k + o) mod m: the reference's (k + o + m) % m wherever that is
// non-negative (src/quasi2DFunctions.cu:260, 265)
inline int q2_wrap(int k, int o, int m) {
  int r = (k + o) % m;
  return r < 0 ? r + m : r;
}

// The node at or below a coordinate (src/quasi2DFunctions.cu:243-252).
inline int q2_node(double r, double invL, double L, double invd, int m) {
  return cellidx(minimage(r, invL, L), invd, m);
}

// Wrapped distance from a coordinate to node k (src/quasi2DFunctions.cu:262-270).
inline double q2_dist(double r, int k, double L, int m, double invL) {
  double d = r - (k * L / m) + L * 0.5;
  return minimage(d, invL, L);
}

// Adds g(r) * (ax, ay) of the stencil of (rx, ry) to the real parts of Z
// (src/quasi2DFunctions.cu:255-281); with drift, -g(r) (kT/var) (dx, dy)
// instead (src/quasi2DFunctions.cu:358-389).
void q2_spread(orc_state* s, double rx, double ry, double ax, double ay, bool drift) {
  const int mx = s->mx, my = s->my, w = s->q2_kw;
  const double lx = s->c.lx, ly = s->c.ly;
  const int kx = q2_node(rx, s->invlx, lx, s->invdx, mx);
  const int ky = q2_node(ry, s->invly, ly, s->invdy, my);
  cplx* Zx = s->Z.data();
  cplx* Zy = s->Z.data() + s->nc;
  for (int ix = -w; ix <= w; ++ix) {
    const int kxn = q2_wrap(kx, ix, mx);
    const double dxr = q2_dist(rx, kxn, lx, mx, s->invlx);
    for (int iy = -w; iy <= w; ++iy) {
      const int kyn = q2_wrap(ky, iy, my);
      const int c = kxn + kyn * mx;
      const double dyr = q2_dist(ry, kyn, ly, my, s->invly);
      const double r2 = dxr * dxr + dyr * dyr;
      if (drift) {
        const double g = gauss2d(r2, s->q2_var) * s->c.temperature / s->q2_var;
        Zx[c] += -g * dxr;
        Zy[c] += -g * dyr;
      } else {
        const double g = gauss2d(r2, s->q2_var);
        Zx[c] += g * ax;
        Zy[c] += g * ay;
      }
    }
  }
}

// u = sum_nodes g(r) v (src/quasi2DFunctions.cu:720-752)
void q2_interp(const orc_state* s, double rx, double ry, double& ux, double& uy) {
  const int mx = s->mx, my = s->my, w = s->q2_kw;
  const double lx = s->c.lx, ly = s->c.ly;
  const int kx = q2_node(rx, s->invlx, lx, s->invdx, mx);
  const int ky = q2_node(ry, s->invly, ly, s->invdy, my);
  const double* vx = s->v.data();
  const double* vy = s->v.data() + s->nc;
  ux = 0.0;
  uy = 0.0;
  for (int ix = -w; ix <= w; ++ix) {
    const int kxn = q2_wrap(kx, ix, mx);
    const double dxr = q2_dist(rx, kxn, lx, mx, s->invlx);
    for (int iy = -w; iy <= w; ++iy) {
      const int kyn = q2_wrap(ky, iy, my);
      const double dyr = q2_dist(ry, kyn, ly, my, s->invly);
      const double g = gauss2d(dxr * dxr + dyr * dyr, s->q2_var);
      ux += g * vx[kxn + kyn * mx];
      uy += g * vy[kxn + kyn * mx];
    }
  }
}

// Bonded (src/quasiNeutrallyBuoyantFunctions2D.cu:201-260) and pair forces
// over the 9 neighbour cells of a 2-D cell list (src/quasi2DFunctions.cu:53-235).
void q2_forces(orc_state* s) {
  const int np = s->np;
  const double* q = s->q.data();
  build_cells(s, q);
  s->F.assign(3 * (size_t)np, 0.0);
  const double c1 = s->c.cutoff > 0 ? 2.0 * s->c.soft_epsilon / s->c.cutoff : 0.0;
  const double c2 = s->c.cutoff > 0 ? 1.0 / s->c.cutoff : 0.0;
  // own cell, -y, -x, +x, +y, then (+x,+y), (+x,-y), (-x,+y), (-x,-y)
  const int order[9][2] = {{0, 0}, {0, -1}, {-1, 0}, {1, 0}, {0, 1}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
#pragma omp parallel for schedule(static)
  for (int i = 0; i < np; ++i) {
    const double rx = q[i], ry = q[np + i];
    double fx = 0.0, fy = 0.0;
    if (s->bonded) {
      for (int j = 0; j < s->bpp_cnt[i]; ++j) {
        const int idx = s->bpp_idx[s->bpp_off[i] + j];
        const double x = q[idx], y = q[np + idx];
        const double r0 = s->bpp_r0[s->bpp_off[i] + j], k = s->bpp_k[s->bpp_off[i] + j];
        if (r0 == 0) {
          fx += -k * (rx - x);
          fy += -k * (ry - y);
        } else {
          const double r = std::sqrt((x - rx) * (x - rx) + (y - ry) * (y - ry));
          if (r > 0) {
            fx += -k * (1 - r0 / r) * (rx - x);
            fy += -k * (1 - r0 / r) * (ry - y);
          }
        }
      }
      for (int j = 0; j < s->bfp_cnt[i]; ++j) {
        const int p = s->bfp_off[i] + j;
        const double x = s->bfp_xyz[3 * p], y = s->bfp_xyz[3 * p + 1];
        const double r0 = s->bfp_r0[p], k = s->bfp_k[p];
        if (r0 == 0) {
          fx += -k * (rx - x);
          fy += -k * (ry - y);
        } else {
          const double r = std::sqrt((x - rx) * (x - rx) + (y - ry) * (y - ry));
          if (r > 0) {
            fx += -k * (1 - r0 / r) * (rx - x);
            fy += -k * (1 - r0 / r) * (ry - y);
          }
        }
      }
    }
    if (s->c.pair != ORC_PAIR_NONE) {
      const int c = s->cell_of[i];
      const int cx = c % s->mnx, cy = c / s->mnx;
      for (int o = 0; o < 9; ++o) {
        const int nx = (cx + order[o][0] + s->mnx) % s->mnx;
        const int ny = (cy + order[o][1] + s->mny) % s->mny;
        const int cc = nx + ny * s->mnx;
        for (int k = s->cstart[cc]; k < s->cstart[cc + 1]; ++k) {
          const int j = s->csorted[k];
          double rxij = rx - q[j];
          rxij = rxij - (double)(int)(rxij * s->invlx + 0.5 * sgn(rxij)) * s->c.lx;
          double ryij = ry - q[np + j];
          ryij = ryij - (double)(int)(ryij * s->invly + 0.5 * sgn(ryij)) * s->c.ly;
          const double r2 = rxij * rxij + ryij * ryij;
          double f;
          if (s->c.pair == ORC_PAIR_TABLE_LJ) {
            f = (double)tex_linear(s->ljtab.data(), 4096, (float)(r2 * s->invcut2));
          } else {
            if (j == i || r2 >= s->c.cutoff * s->c.cutoff || r2 == 0.0) continue;
            f = c1 * (1.0 / std::sqrt(r2) - c2);
          }
          fx += f * rxij;
          fy += f * ryij;
        }
      }
    }
    s->F[i] = fx;
    s->F[np + i] = fy;
  }
}

// Wave numbers of mode i for the deterministic updates
// (src/quasi2DFunctions.cu:402-423): signed, with the Nyquist rows folded.
inline void q2_k_det(const orc_state* s, int i, double& kx, double& ky) {
  const int mx = s->mx, my = s->my;
  int wy = i / mx, wx = i % mx;
  if (wx > mx / 2) wx -= mx;
  if (wy > my / 2) wy -= my;
  const bool xHalf = (mx % 2) == 0 && (wx == mx / 2);
  const bool yHalf = (my % 2) == 0 && (wy == my / 2);
  if (xHalf && wy < 0) wx *= -1;
  else if (yHalf && wx < 0) wy *= -1;
  const double pi = 3.1415926535897932385;
  kx = wx * 2 * pi / s->c.lx;
  ky = wy * 2 * pi / s->c.ly;
}

// Noise bookkeeping of mode i (src/quasi2DFunctions.cu:598-635): the
// canonical |wave numbers|, the noise index shared by i and -i, and whether
// the imaginary part flips (the conjugate partner).
struct Q2Mode {
  double kx, ky;
  int index;
  bool xHalf, yHalf, flip;
  int wx, wy;
};
inline Q2Mode q2_mode_noise(const orc_state* s, int i) {
  const int mx = s->mx, my = s->my, nModes = s->nc + mx + my;
  Q2Mode m;
  int wy = i / mx, wx = i % mx, fx = wx, fy = wy, shift = 0;
  if (wx > mx / 2) {
    fx = wx - mx;
    wx = mx - wx;
  }
  if (wy > my / 2) {
    fy = wy - my;
    wy = my - wy;
  }
  m.xHalf = (mx % 2) == 0 && (wx == mx / 2);
  m.yHalf = (my % 2) == 0 && (wy == my / 2);
  if (m.xHalf && fy < 0) fx *= -1;
  else if (m.yHalf && fx < 0) fy *= -1;
  const double pi = 3.1415926535897932385;
  m.kx = wx * 2 * pi / s->c.lx;
  m.ky = wy * 2 * pi / s->c.ly;
  if (fx * fy < 0) {
    shift = nModes / 2;
    m.kx *= -1.0;
  }
  m.index = wy * mx + wx + shift;
  m.flip = (fx < 0) || (fx == 0 && fy < 0);
  m.wx = wx;
  m.wy = wy;
  return m;
}

// Fourier-space solve plus stochastic velocity of every mode.
void q2_fourier(orc_state* s) {
  const int nc = s->nc, mx = s->mx, my = s->my, nModes = nc + mx + my;
  const double eta = s->c.shearviscosity, pi_half_inv = 0.56418958354775628695;
  const double sigma = std::sqrt(s->q2_var), prefactor = s->q2_fact1;
  const double* R = s->noise.data();
  cplx* Zx = s->Z.data();
  cplx* Zy = s->Z.data() + nc;
  const bool rpy = s->c.scheme == ORC_SCHEME_QUASI2D;
  const double kc = s->c.saffman_kc, lw = s->c.saffman_width;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nc; ++i) {
    // deterministic part
    double kx, ky;
    q2_k_det(s, i, kx, ky);
    const double vxr = Zx[i].real(), vxi = Zx[i].imag(), vyr = Zy[i].real(), vyi = Zy[i].imag();
    double oxr = 0, oxi = 0, oyr = 0, oyi = 0;
    if (i != 0) {
      if (rpy) {
        // src/quasi2DFunctions.cu:450-510
        const double k_inv = 1.0 / std::sqrt(kx * kx + ky * ky);
        const double k3_inv = k_inv * k_inv * k_inv;
        const double k = 1.0 / k_inv, kn = sigma * k;
        const double f = 0.5 * (std::erfc(kn) * (0.5 + kn * kn) * std::exp(kn * kn) - pi_half_inv * kn);
        const double g = 0.5 * std::erfc(kn) * std::exp(kn * kn);
        oxr = (k3_inv / eta) * (g * ky * (ky * vxr - kx * vyr) + f * kx * (kx * vxr + ky * vyr));
        oxi = (k3_inv / eta) * (g * ky * (ky * vxi - kx * vyi) + f * kx * (kx * vxi + ky * vyi));
        oyr = (k3_inv / eta) * (g * (-kx) * (ky * vxr - kx * vyr) + f * ky * (kx * vxr + ky * vyr));
        oyi = (k3_inv / eta) * (g * (-kx) * (ky * vxi - kx * vyi) + f * ky * (kx * vxi + ky * vyi));
      } else {
        // src/quasi2DFunctions.cu:767-827 (Stokes) and 966-1035 (Saffman)
        const double L = -(kx * kx) - (ky * ky);
        double den;
        if (kc != 0.0) {
          const double kmod = std::sqrt(-L);
          const double corr = lw != 0.0 ? std::tanh(kmod * lw) : 1.0;
          den = eta * (kmod * (kmod + kc * corr));
        } else {
          den = -eta * L;
        }
        const double GWr = kx * vxr + ky * vyr, GWi = kx * vxi + ky * vyi;
        oxr = (vxr + kx * GWr / L) / den;
        oxi = (vxi + kx * GWi / L) / den;
        oyr = (vyr + ky * GWr / L) / den;
        oyi = (vyi + ky * GWi / L) / den;
      }
    }
    // stochastic part
    const Q2Mode m = q2_mode_noise(s, i);
    double Wxr = 0, Wxi = 0, Wyr = 0, Wyi = 0;
    const double mkx = m.kx, mky = m.ky;
    const bool edge = (m.xHalf && m.wy == 0) || (m.yHalf && m.wx == 0) || (m.xHalf && m.yHalf);
    if (rpy) {
      // src/quasi2DFunctions.cu:590-678 (factorScheme 1)
      if (i != 0) {
        const double k = std::sqrt(mkx * mkx + mky * mky);
        const double k3half_inv = 1.0 / std::sqrt(k * k * k);
        const double kn = sigma * k;
        const double f_half =
            std::sqrt(0.5 * (std::erfc(kn) * (0.5 + kn * kn) * std::exp(kn * kn) - pi_half_inv * kn));
        const double g_half = std::sqrt(0.5 * std::erfc(kn) * std::exp(kn * kn));
        const double a = g_half * mky, b = f_half * mkx, c = g_half * (-mkx), d = f_half * mky;
        if (edge) {
          Wxr = std::sqrt(2.0) * prefactor * k3half_inv * (a * R[m.index] + b * R[nModes + m.index]);
          Wyr = std::sqrt(2.0) * prefactor * k3half_inv * (c * R[m.index] + d * R[nModes + m.index]);
        } else {
          Wxr = prefactor * k3half_inv * (a * R[m.index] + b * R[nModes + m.index]);
          Wyr = prefactor * k3half_inv * (c * R[m.index] + d * R[nModes + m.index]);
          Wxi = prefactor * k3half_inv * (a * R[nModes * 2 + m.index] + b * R[nModes * 3 + m.index]);
          Wyi = prefactor * k3half_inv * (c * R[nModes * 2 + m.index] + d * R[nModes * 3 + m.index]);
        }
      }
    } else {
      // src/quasi2DFunctions.cu:829-904 (Stokes) and 1037-1119 (Saffman)
      const bool nyq = ((mx % 2) == 0 && (m.wx == mx / 2)) || ((my % 2) == 0 && (m.wy == my / 2)) || i == 0;
      if (!nyq) {
        double amp;
        if (kc != 0.0) {
          const double kmod2 = mkx * mkx + mky * mky, kmod = std::sqrt(kmod2);
          const double corr = lw != 0.0 ? std::tanh(kmod * lw) : 1.0;
          amp = 1.0 / std::sqrt(kmod * kmod2 * (kmod + kc * corr));
        } else {
          amp = 1.0 / (mkx * mkx + mky * mky);
        }
        if (edge) {
          Wxr = std::sqrt(2.0) * prefactor * amp * (mky * R[m.index]);
          Wyr = std::sqrt(2.0) * prefactor * amp * ((-mkx) * R[m.index]);
        } else {
          Wxr = prefactor * amp * (mky * R[m.index]);
          Wyr = prefactor * amp * ((-mkx) * R[m.index]);
          Wxi = prefactor * amp * (mky * R[nModes * 2 + m.index]);
          Wyi = prefactor * amp * ((-mkx) * R[nModes * 2 + m.index]);
        }
      }
    }
    if (m.flip) {
      Wxi = -Wxi;
      Wyi = -Wyi;
    }
    Zx[i] = cplx(oxr + Wxr, oxi + Wxi);
    Zy[i] = cplx(oyr + Wyr, oyi + Wyi);
  }
}

// One step of runSchemeQuasi2D (src/runSchemeQuasi2D.cu:108-250).
void one_step_q2d(orc_state* s) {
  const int np = s->np, nc = s->nc, mx = s->mx, my = s->my;
  {
    const size_t n = (size_t)4 * (nc + mx + my) + (size_t)2 * np * s->c.ndrift;
    s->noise.resize(n);
    for (size_t k = 0; k < n; ++k) s->noise[k] = philox_normal(s->c.seed, s->t, k);
  }
  std::fill(s->Z.begin(), s->Z.end(), cplx(0, 0));
  const double* q = s->q.data();
  if (s->c.nonbonded) {
    q2_forces(s);
    for (int i = 0; i < np; ++i) q2_spread(s, q[i], q[np + i], s->F[i], s->F[np + i], false);
  }
  if (s->c.use_rfd)
    for (int i = 0; i < np; ++i) q2_spread(s, q[i], q[np + i], 0.0, 0.0, true);
  if (s->c.shear_amp != 0.0) {
    // src/quasi2DFunctions.cu:3-12
    const double pi2 = 2.0 * 3.1415926535897932385;
    for (int i = 0; i < nc; ++i)
      s->Z[nc + i] += s->c.shear_amp * std::sin(pi2 * ((i % mx) / (double)mx));
  }
  for (int comp = 0; comp < 2; ++comp)
    fft3d(s->Z.data() + (size_t)comp * nc, mx, my, 1, s->Px, s->Py, s->Pz, -1);
  q2_fourier(s);
  for (int comp = 0; comp < 2; ++comp)
    fft3d(s->Z.data() + (size_t)comp * nc, mx, my, 1, s->Px, s->Py, s->Pz, +1);
  for (size_t k = 0; k < (size_t)2 * nc; ++k) s->v[k] = s->Z[k].real() / (double)nc;
  // src/quasi2DFunctions.cu:681-760: q' = q + dx dy dt J(position) v
  const double vol = s->dx * s->dy, dt = s->c.dt;
  if (s->c.predictor_corrector) {
    for (int i = 0; i < np; ++i) {
      double ux, uy;
      q2_interp(s, s->q[i], s->q[np + i], ux, uy);
      s->qp[i] = s->q[i] + vol * ux * (0.5 * dt);
      s->qp[np + i] = s->q[np + i] + vol * uy * (0.5 * dt);
    }
    for (int i = 0; i < np; ++i) {
      double ux, uy;
      q2_interp(s, s->qp[i], s->qp[np + i], ux, uy);
      s->q[i] = s->q[i] + vol * ux * dt;
      s->q[np + i] = s->q[np + i] + vol * uy * dt;
    }
  } else {
    for (int i = 0; i < np; ++i) {
      double ux, uy;
      q2_interp(s, s->q[i], s->q[np + i], ux, uy);
      s->q[i] = s->q[i] + vol * ux * dt;
      s->q[np + i] = s->q[np + i] + vol * uy * dt;
    }
  }
  s->t++;
}

}  // namespace

// ================================================================== C ABI ==
extern "C" {

orc_state* orc_create(const orc_config* cfg, int64_t np, const double* q) {
  if (!cfg || cfg->mx <= 0 || cfg->my <= 0 || cfg->mz <= 0 || np < 0) return nullptr;
  orc_state* s = new orc_state();
  s->c = *cfg;
  s->mx = cfg->mx;
  s->my = cfg->my;
  s->mz = cfg->mz;
  s->nc = s->mx * s->my * s->mz;
  s->dx = cfg->lx / (double)s->mx;
  s->dy = cfg->ly / (double)s->my;
  s->dz = cfg->lz / (double)s->mz;
  s->invdx = (double)s->mx / cfg->lx;
  s->invdy = (double)s->my / cfg->ly;
  s->invdz = (double)s->mz / cfg->lz;
  s->invlx = 1. / cfg->lx;
  s->invly = 1. / cfg->ly;
  s->invlz = 1. / cfg->lz;
  s->dV = s->dx * s->dy * s->dz;
  double T = cfg->temperature, eta = cfg->shearviscosity, dt = cfg->dt;
  s->fact1 = std::sqrt((4. * T * eta) / (s->dV * dt));
  s->fact4 = std::sqrt((2. * T * eta) / (s->dV * dt));
  if (cfg->scheme == ORC_SCHEME_INCOMPRESSIBLE) {
    // src/createCellsIncompressibleGPU.cu:60-63
    const double rho = cfg->density;
    s->fact1 = std::sqrt((4. * T * eta * dt) / (s->dV * rho * rho));
    s->fact4 = std::sqrt((2. * T * eta * dt) / (s->dV * rho * rho));
  }
  s->fact2 = std::sqrt(T * cfg->extra_mobility * dt);
  s->Px.init(s->mx);
  s->Py.init(s->my);
  s->Pz.init(s->mz);
  const int m[3] = {s->mx, s->my, s->mz};
  const double invd[3] = {s->invdx, s->invdy, s->invdz};
  double pi = 4. * std::atan(1.);
  for (int a = 0; a < 3; ++a) {
    s->gradK[a].resize(m[a]);
    s->expKre[a].resize(m[a]);
    s->expKim[a].resize(m[a]);
    for (int j = 0; j < m[a]; ++j) {
      s->gradK[a][j] = 2 * invd[a] * std::sin(pi * j / double(m[a]));
      s->expKre[a][j] = std::cos(pi * j / double(m[a]));
      s->expKim[a][j] = std::sin(pi * j / double(m[a]));
    }
  }
  if (cfg->cutoff > 0) {
    s->mnx = std::max(3, (int)(cfg->lx / cfg->cutoff));
    s->mny = std::max(3, (int)(cfg->ly / cfg->cutoff));
    s->mnz = std::max(3, (int)(cfg->lz / cfg->cutoff));
    s->invcut2 = 1. / (cfg->cutoff * cfg->cutoff);
  } else {
    s->mnx = s->mny = s->mnz = 3;
    s->invcut2 = 0.0;
  }
  if (cfg->scheme == ORC_SCHEME_QUASI2D || cfg->scheme == ORC_SCHEME_STOKES2D) {
    // src/createBoundariesQuasi2DGPU.cu:89-93: int(L / rc) cells per side
    // (the callers keep at least 3), one layer in z
    if (cfg->cutoff > 0) {
      s->mnx = (int)(cfg->lx / cfg->cutoff);
      s->mny = (int)(cfg->ly / cfg->cutoff);
    }
    s->mnz = 1;
    // src/createCellsQuasi2DGPU.cu:49-79
    const double a = cfg->radius;
    s->q2_var = cfg->scheme == ORC_SCHEME_QUASI2D ? std::pow(a / std::sqrt(3.1415926535897932385), 2)
                                                  : std::pow(a * 0.66556976637237890625, 2);
    s->q2_kw = (int)(3.0 * a * s->mx / cfg->lx) + 1;
    if (s->q2_kw > s->mx / 2) s->q2_kw = s->mx / 2;
    s->q2_fact1 = std::sqrt(1.0 * cfg->temperature / (cfg->shearviscosity * cfg->dt * cfg->lx * cfg->ly)) *
                  (s->mx * s->my * s->mz);
  }
  s->mN = s->mnx * s->mny * s->mnz;
  if (cfg->pair == ORC_PAIR_TABLE_LJ) build_ljtable(s);
  s->np = (int)np;
  s->q.assign(q, q + 3 * (size_t)np);
  s->qp = s->q;
  s->F.assign(3 * (size_t)np, 0.0);
  s->f.assign(3 * (size_t)s->nc, 0.0);
  s->v.assign(3 * (size_t)s->nc, 0.0);
  s->acc.assign(3 * (size_t)s->nc, 0.0);
  s->Z.assign(3 * (size_t)s->nc, cplx(0, 0));
  s->bpp_cnt.assign(np, 0);
  s->bpp_off.assign(np, 0);
  s->bfp_cnt.assign(np, 0);
  s->bfp_off.assign(np, 0);
  return s;
}

void orc_destroy(orc_state* s) { delete s; }

// Directed entries: entry b acts on particle bi[b] only, as a line of the
// old bond-file format (bondedForcesVersion 1) does; the CSR groups the
// entries by bi in their order, which for the sorted files the reference
// accepts is its own CSR (src/initializeBondedForcesOldVersion.cpp:41-238).
// Tethers as in orc_set_bonds.
static int set_bonds_csr(orc_state* s, int64_t nbonds, const int32_t* bi, const int32_t* bj,
                         const double* bk, const double* br0, int64_t nfixed, const int32_t* fi,
                         const double* fk, const double* fr0, const double* fxyz, bool directed) {
  int np = s->np;
  for (int64_t b = 0; b < nbonds; ++b)
    if (bi[b] < 0 || bi[b] >= np || bj[b] < 0 || bj[b] >= np) return -1;
  for (int64_t b = 0; b < nfixed; ++b)
    if (fi[b] < 0 || fi[b] >= np) return -1;
  const int64_t nent = directed ? nbonds : 2 * nbonds;
  s->bpp_cnt.assign(np, 0);
  s->bfp_cnt.assign(np, 0);
  for (int64_t b = 0; b < nbonds; ++b) {
    s->bpp_cnt[bi[b]]++;
    if (!directed) s->bpp_cnt[bj[b]]++;
  }
  for (int64_t b = 0; b < nfixed; ++b) s->bfp_cnt[fi[b]]++;
  s->bpp_off.assign(np, 0);
  s->bfp_off.assign(np, 0);
  for (int i = 1; i < np; ++i) {
    s->bpp_off[i] = s->bpp_off[i - 1] + s->bpp_cnt[i - 1];
    s->bfp_off[i] = s->bfp_off[i - 1] + s->bfp_cnt[i - 1];
  }
  s->bpp_idx.assign(nent, 0);
  s->bpp_k.assign(nent, 0.0);
  s->bpp_r0.assign(nent, 0.0);
  std::vector<int> tmp(np, 0);
  for (int64_t b = 0; b < nbonds; ++b) {
    int i1 = bi[b], i2 = bj[b];
    int p1 = s->bpp_off[i1] + tmp[i1]++;
    s->bpp_idx[p1] = i2;
    s->bpp_k[p1] = bk[b];
    s->bpp_r0[p1] = br0[b];
    if (directed) continue;
    int p2 = s->bpp_off[i2] + tmp[i2]++;
    s->bpp_idx[p2] = i1;
    s->bpp_k[p2] = bk[b];
    s->bpp_r0[p2] = br0[b];
  }
  std::fill(tmp.begin(), tmp.end(), 0);
  s->bfp_k.assign(nfixed, 0.0);
  s->bfp_r0.assign(nfixed, 0.0);
  s->bfp_xyz.assign(3 * nfixed, 0.0);
  for (int64_t b = 0; b < nfixed; ++b) {
    int i1 = fi[b];
    int p = s->bfp_off[i1] + tmp[i1];
    s->bfp_k[p] = fk[b];
    s->bfp_r0[p] = fr0[b];
    s->bfp_xyz[3 * p] = fxyz[3 * b];
    s->bfp_xyz[3 * p + 1] = fxyz[3 * b + 1];
    s->bfp_xyz[3 * p + 2] = fxyz[3 * b + 2];
    tmp[i1]++;
  }
  s->bonded = (nbonds + nfixed) > 0;
  return 0;
}

int orc_set_bonds(orc_state* s, int64_t nbonds, const int32_t* bi, const int32_t* bj,
                  const double* bk, const double* br0, int64_t nfixed, const int32_t* fi,
                  const double* fk, const double* fr0, const double* fxyz) {
  // CSR exactly as src/initializeBondedForces.cpp:31-150: both endpoints
  // store each particle-particle bond, in file order.
  return set_bonds_csr(s, nbonds, bi, bj, bk, br0, nfixed, fi, fk, fr0, fxyz, false);
}

int orc_set_bonds_directed(orc_state* s, int64_t nentries, const int32_t* bi, const int32_t* bj,
                           const double* bk, const double* br0, int64_t nfixed, const int32_t* fi,
                           const double* fk, const double* fr0, const double* fxyz) {
  return set_bonds_csr(s, nentries, bi, bj, bk, br0, nfixed, fi, fk, fr0, fxyz, true);
}

int orc_step(orc_state* s, int64_t nsteps) {
  for (int64_t k = 0; k < nsteps; ++k) one_step(s);
  return 0;
}

void orc_set_velocity(orc_state* s, const double* v) {
  const size_t n3 = 3 * (size_t)s->nc;
  for (size_t k = 0; k < n3; ++k) s->Z[k] = cplx(v[k], 0.0);
  inc_transform(s, -1);
  inc_fourier(s, false);
  inc_transform(s, +1);
  for (size_t k = 0; k < n3; ++k) s->v[k] = s->Z[k].real() / (double)s->nc;
}

void orc_get_positions(const orc_state* s, double* out) {
  std::memcpy(out, s->q.data(), sizeof(double) * 3 * (size_t)s->np);
}
void orc_set_positions(orc_state* s, const double* in) {
  std::memcpy(s->q.data(), in, sizeof(double) * 3 * (size_t)s->np);
}
void orc_get_predictor(const orc_state* s, double* out) {
  std::memcpy(out, s->qp.data(), sizeof(double) * 3 * (size_t)s->np);
}
void orc_get_forces(const orc_state* s, double* out) {
  std::memcpy(out, s->F.data(), sizeof(double) * 3 * (size_t)s->np);
}
void orc_get_velocity(const orc_state* s, double* out) {
  std::memcpy(out, s->v.data(), sizeof(double) * 3 * (size_t)s->nc);
}
uint64_t orc_get_step(const orc_state* s) { return s->t; }
void orc_set_step(orc_state* s, uint64_t t) { s->t = t; }
int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_noise(uint64_t seed, uint64_t t, uint64_t first, int64_t count, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < count; ++k) out[k] = philox_normal(seed, t, first + (uint64_t)k);
}

int orc_neighbor_grid(const orc_state* s, int32_t* dims3) {
  dims3[0] = s->mnx;
  dims3[1] = s->mny;
  dims3[2] = s->mnz;
  return s->mN;
}

void orc_cell_list(orc_state* s, const double* q, int32_t* cell_of, int32_t* start,
                   int32_t* sorted) {
  build_cells(s, q);
  for (int i = 0; i < s->np; ++i) {
    cell_of[i] = s->cell_of[i];
    sorted[i] = s->csorted[i];
  }
  for (int c = 0; c <= s->mN; ++c) start[c] = s->cstart[c];
}

void orc_forces(orc_state* s, const double* q, double* F) {
  build_cells(s, q);
  compute_forces(s, q, F);
}

void orc_spread(orc_state* s, const double* q, const double* F, double* f) {
  std::fill(s->f.begin(), s->f.end(), 0.0);
  spread_add(s, q, q, F);
  std::memcpy(f, s->f.data(), sizeof(double) * 3 * (size_t)s->nc);
}

void orc_solve(orc_state* s, const double* W, double* v) {
  for (size_t k = 0; k < (size_t)3 * s->nc; ++k) s->Z[k] = cplx(W[k], 0.0);
  solve(s);
  std::memcpy(v, s->v.data(), sizeof(double) * 3 * (size_t)s->nc);
}

void orc_interp(orc_state* s, const double* q, const double* v, double* u) {
  interpolate(s, q, v, u);
}

void orc_build_W(orc_state* s, const double* f, int second, double* W) {
  // W for draw s->t, from a given spread field f (3 nc)
  draw_noise(s);
  std::memcpy(s->f.data(), f, sizeof(double) * 3 * (size_t)s->nc);
  construct_W(s, second ? std::sqrt(0.5) : std::sqrt(2.0), second != 0);
  for (size_t k = 0; k < (size_t)3 * s->nc; ++k) W[k] = s->Z[k].real();
}

void orc_fft3d(int mx, int my, int mz, int sign, double* re_im) {
  Plan1D Px, Py, Pz;
  Px.init(mx);
  Py.init(my);
  Pz.init(mz);
  fft3d(reinterpret_cast<cplx*>(re_im), mx, my, mz, Px, Py, Pz, sign);
}

void orc_ljtable(orc_state* s, float* out) {
  if (s->ljtab.empty()) build_ljtable(s);
  std::memcpy(out, s->ljtab.data(), sizeof(float) * 4096);
}

float orc_tex_linear(const float* table, int n, float x) { return tex_linear(table, n, x); }

double orc_delta3(double x) { return delta3(x); }
double orc_delta4(double x) { return delta4(x); }

}  // extern "C"
