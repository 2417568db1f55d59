// fsl_group.cu -- slots, size-class groups and the graph-captured step of
// any number of groups (declared in fsl_group.cuh).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "fsl_group.cuh"

namespace fsl {

static_assert((int)PREC_FIXED == (int)FSL_PRECISION_FIXED64 &&
                  (int)PREC_FLOAT == (int)FSL_PRECISION_FLOAT_ATOMIC &&
                  (int)PREC_F64 == (int)FSL_PRECISION_FP64,
              "precision codes");

namespace {
thread_local char g_msg[512] = "";

constexpr size_t kAlign = 256;
size_t align_up(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }

// Byte offsets of one slot's buffers inside its arena.
struct SlotLayout {
  size_t q, qp, F, u, qw, ws, cell_of, tmp, sorted, bpp_cnt, bpp_off, bfp_cnt, bfp_off, cnt, fill, start,
      bsum, ljtab, noise, ndiv, stc, grid, spec, v, wbuf, noise64, v64, z64, err, t, q0, obs, obs_part, obs_ticket,
      start1, sorted1, ws1, vl_cnt, vl_idx, qref, vl_flag, bar, total;
};

SlotLayout layout(const Params& P, int np_cap) {
  SlotLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += align_up(std::max<size_t>(bytes, 1));
    return o;
  };
  const size_t np = (size_t)np_cap, nc = (size_t)P.nc;
  const size_t mN = (size_t)P.mN;
  const uint64_t noise = (noise_count(P, np_cap) + 3) / 4 * 4;
  L.q = take(sizeof(double) * 3 * np);
  L.qp = take(sizeof(double) * 3 * np);
  L.F = take(sizeof(double) * 3 * np);
  L.u = take(sizeof(double) * 3 * np);
  L.qw = take(sizeof(double) * 3 * np);
  L.ws = take(sizeof(double) * 3 * np);
  L.cell_of = take(sizeof(int) * np);
  L.tmp = take(sizeof(int) * np);
  L.sorted = take(sizeof(int) * np);
  L.bpp_cnt = take(sizeof(int) * np);
  L.bpp_off = take(sizeof(int) * np);
  L.bfp_cnt = take(sizeof(int) * np);
  L.bfp_off = take(sizeof(int) * np);
  L.cnt = take(sizeof(int) * mN);
  L.fill = take(sizeof(int) * mN);
  L.start = take(sizeof(int) * (mN + 1));
  L.bsum = take(sizeof(int) * std::max<size_t>((mN + 4095) / 4096 + 1, kCoopMaxBlocks + 1));
  L.ljtab = take(sizeof(float) * kLjTableSize);
  // the FP32 field buffers, or their FP64 counterparts (the spread field has
  // 8-byte entries in every form: fixed point, or FP64; the float-atomic
  // form uses its first 3 nc floats)
  const bool f64 = P.prec == FSL_PRECISION_FP64;
  L.noise = take(f64 ? 0 : sizeof(float) * noise);
  // the stress divergence D1 | D12 of the 3-D Stokes schemes (k_div)
  L.ndiv = take(!f64 && P.scheme <= FSL_SCHEME_FIRST_ORDER ? sizeof(float) * 6 * nc : 0);
  // the midpoint scheme's stencil cache: every spread stores the nodes and
  // weights of its quads for the interpolation at the same positions
  // (3 x 16 bytes per lane, 4 lanes per particle)
  L.stc = take(!f64 && P.scheme == FSL_SCHEME_MIDPOINT ? sizeof(uint4) * 3 * 4 * np : 0);
  L.grid = take(sizeof(unsigned long long) * 3 * nc);
  L.spec = take(f64 ? 0 : sizeof(float2) * 3 * (size_t)P.my * P.mz * P.mxh);
  L.v = take(f64 ? 0 : sizeof(float) * 3 * nc);
  L.wbuf = take(f64 ? 0 : sizeof(float) * 3 * nc);
  L.noise64 = take(f64 ? sizeof(double) * noise : 0);
  L.v64 = take(f64 ? sizeof(double) * 3 * nc : 0);
  L.z64 = take(f64 ? sizeof(double2) * 3 * nc : 0);
  L.err = take(sizeof(int) * 4);
  L.t = take(sizeof(uint64_t));
  L.q0 = take(P.observe ? sizeof(double) * 3 * np : 0);
  L.obs = take(sizeof(double) * kObsSlots);
  L.obs_part = take(P.observe ? sizeof(double) * kObsVals * kObsMaxBlocks : 0);
  L.obs_ticket = take(sizeof(unsigned));
  // the 3-D Stokes schemes build two cell lists per step and keep both
  const bool two_lists = P.scheme <= FSL_SCHEME_FIRST_ORDER;
  L.start1 = take(two_lists ? sizeof(int) * (mN + 1) : 0);
  L.sorted1 = take(two_lists ? sizeof(int) * np : 0);
  L.ws1 = take(two_lists ? sizeof(double) * 3 * np : 0);
  L.vl_cnt = take(P.verlet ? sizeof(int) * np : 0);
  L.vl_idx = take(P.verlet ? sizeof(int) * (size_t)kVlCap * np : 0);
  L.qref = take(P.verlet ? sizeof(double) * 3 * np : 0);
  L.vl_flag = take(sizeof(uint64_t) * 3);
  L.bar = take(sizeof(unsigned) * 2);
  L.total = off;
  return L;
}

bool factor_ok(int n) {
  if (n < 3) return false;
  const int ps[5] = {2, 3, 5, 7, 11};
  for (int p : ps)
    while (n % p == 0) n /= p;
  return n == 1;
}
}  // namespace

int errorf(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
  return code;
}

const char* last_error() { return g_msg; }

int set_last_error(int code, const char* msg) { return errorf(code, "%s", msg); }

int cuda_fail(cudaError_t e, const char* what) {
  cudaGetLastError();
  return errorf(e == cudaErrorMemoryAllocation ? FSL_E_NOMEM : FSL_E_CUDA, "%s: %s", what,
                cudaGetErrorString(e));
}

bool ClassKey::operator<(const ClassKey& o) const {
  const int a[10] = {mx, my, mz, mnx, mny, mnz, kernel, scheme, prec, observe};
  const int b[10] = {o.mx, o.my, o.mz, o.mnx, o.mny, o.mnz, o.kernel, o.scheme, o.prec, o.observe};
  return std::lexicographical_compare(a, a + 10, b, b + 10);
}
bool ClassKey::operator==(const ClassKey& o) const { return !(*this < o) && !(o < *this); }

ClassKey class_of(const Params& P) {
  return ClassKey{P.mx, P.my, P.mz, P.mnx, P.mny, P.mnz, P.kernel, P.scheme, P.prec, P.observe};
}

int make_params(const fsl_config& c, int64_t np, Params& P) {
  if (c.scheme < 0 || c.scheme > 4) return errorf(FSL_E_ARG, "unknown scheme %d", c.scheme);
  const bool two_d = c.scheme == FSL_SCHEME_QUASI2D || c.scheme == FSL_SCHEME_STOKES2D;
  const bool incomp = c.scheme == FSL_SCHEME_INCOMPRESSIBLE;
  if (incomp && np != 0) return errorf(FSL_E_ARG, "the incompressible scheme has no particles");
  if (incomp && !(c.density > 0)) return errorf(FSL_E_ARG, "densfluid must be > 0");
  if (two_d && c.mz != 1) return errorf(FSL_E_ARG, "the quasi-2D schemes need cells mx my 1");
  if (c.mx < 3 || c.my < 3 || (!two_d && c.mz < 3))
    return errorf(FSL_E_ARG, "cells must be >= 3 in every direction");
  if (!factor_ok(c.mx) || !factor_ok(c.my) || (!two_d && !factor_ok(c.mz)))
    return errorf(FSL_E_ARG, "cells %d %d %d: every extent must factor into 2,3,5,7,11", c.mx, c.my,
                  c.mz);
  if (c.mx > 1024 || c.my > 1024 || c.mz > 1024)
    return errorf(FSL_E_ARG, "cells per direction limited to 1024");
  if (!(c.lx > 0 && c.ly > 0 && c.lz > 0)) return errorf(FSL_E_ARG, "celldimension must be > 0");
  if (!(c.dt > 0)) return errorf(FSL_E_ARG, "dt must be > 0");
  if (!(c.shearviscosity > 0)) return errorf(FSL_E_ARG, "shearviscosity must be > 0");
  if (!(c.temperature >= 0)) return errorf(FSL_E_ARG, "temperature must be >= 0");
  if (c.kernel != 3 && c.kernel != 4) return errorf(FSL_E_ARG, "kernel must be 3 or 4");
  if (c.pair < 0 || c.pair > 2) return errorf(FSL_E_ARG, "unknown pair potential %d", c.pair);
  if (c.rfd < 0 || c.rfd > 1) return errorf(FSL_E_ARG, "unknown rfd mode %d", c.rfd);
  if (c.precision < 0 || c.precision > 2)
    return errorf(FSL_E_ARG, "unknown precision form %d", c.precision);
  if (c.extra_mobility < 0) return errorf(FSL_E_ARG, "extraMobility must be >= 0");
  if (c.observables != 0 && c.observables != 1) return errorf(FSL_E_ARG, "observables must be 0 or 1");
  if (c.observables && c.scheme > FSL_SCHEME_FIRST_ORDER)
    return errorf(FSL_E_ARG, "observables: 3-D Stokes schemes only");
  if (np < 0 || np > (int64_t)1 << 28) return errorf(FSL_E_ARG, "bad particle count");
  bool pairs = c.nonbonded && c.pair != FSL_PAIR_NONE && np > 0;
  if (pairs && !(c.cutoff > 0)) return errorf(FSL_E_ARG, "cutoff must be > 0 with pair forces");
  int64_t nc64 = (int64_t)c.mx * c.my * c.mz;
  if (nc64 > ((int64_t)1 << 30)) return errorf(FSL_E_ARG, "grid too large");

  std::memset(&P, 0, sizeof(P));
  P.mx = c.mx;
  P.my = c.my;
  P.mz = c.mz;
  P.mxh = c.mx / 2 + 1;
  P.nc = (int)nc64;
  P.lx = c.lx;
  P.ly = c.ly;
  P.lz = c.lz;
  // src/createCellsStokesLimitGPU.cu:71-91
  P.dx = c.lx / double(c.mx);
  P.dy = c.ly / double(c.my);
  P.dz = c.lz / double(c.mz);
  P.invdx = double(c.mx) / c.lx;
  P.invdy = double(c.my) / c.ly;
  P.invdz = double(c.mz) / c.lz;
  P.invlx = 1. / c.lx;
  P.invly = 1. / c.ly;
  P.invlz = 1. / c.lz;
  P.dV = P.dx * P.dy * P.dz;
  P.observe = c.observables;
  // src/createBoundariesRK2GPU.cu:134-141
  if (c.cutoff > 0) {
    P.mnx = std::max(3, (int)(c.lx / c.cutoff));
    P.mny = std::max(3, (int)(c.ly / c.cutoff));
    P.mnz = std::max(3, (int)(c.lz / c.cutoff));
  } else {
    P.mnx = P.mny = P.mnz = 3;
  }
  if ((int64_t)P.mnx * P.mny * P.mnz > ((int64_t)1 << 28))
    return errorf(FSL_E_ARG, "cutoff too small for the box (neighbour grid too large)");
  if (two_d) {
    // src/createBoundariesQuasi2DGPU.cu:89-93: int(L / rc) cells per side in
    // the plane (no lower bound: with fewer than 3 the 9-cell sweep visits a
    // cell more than once, as the reference does), one layer
    if (c.cutoff > 0) {
      P.mnx = (int)(c.lx / c.cutoff);
      P.mny = (int)(c.ly / c.cutoff);
    }
    P.mnz = 1;
    if (c.nonbonded && np > 0 && (P.mnx < 1 || P.mny < 1))
      return errorf(FSL_E_ARG, "cutoff larger than the box");
    // without pair forces the cell list is unused; keep its extents valid
    P.mnx = std::max(P.mnx, 1);
    P.mny = std::max(P.mny, 1);
    if (!(c.radius > 0)) return errorf(FSL_E_ARG, "hydrodynamicRadius must be > 0");
    if (c.ndrift < 0) return errorf(FSL_E_ARG, "nDrift must be >= 0");
  }
  P.mN = P.mnx * P.mny * P.mnz;
  if ((int64_t)((P.mN + 4095) / 4096) > 4096) return errorf(FSL_E_ARG, "neighbour grid too large");
  P.invdnx = double(P.mnx) / c.lx;
  P.invdny = double(P.mny) / c.ly;
  P.invdnz = double(P.mnz) / c.lz;
  P.np = (int)np;
  P.kernel = c.kernel;
  P.pair = c.pair;
  P.nonbonded = c.nonbonded ? 1 : 0;
  P.rfd = c.rfd;
  P.scheme = c.scheme;
  P.prec = c.precision;
  P.bonded = 0;
  P.has_extra = c.extra_mobility != 0.0;
  P.cutoff = c.cutoff;
  P.cutoff2 = c.cutoff * c.cutoff;
  P.invcut2 = c.cutoff > 0 ? 1. / (c.cutoff * c.cutoff) : 0.0;
  P.soft_eps = c.soft_epsilon;
  // 3-D Stokes schemes: soft repulsion through a Verlet list (when the
  // neighbour cells are at least rc wide, so that the list holds exactly
  // the reference's pair set; skin <= 2 cells - rc keeps the list build
  // within two cells), no list at all without pair forces.
  // FLUAMSL_VERLET=0 keeps soft repulsion on the cell-list kernel.
  if (c.scheme <= FSL_SCHEME_FIRST_ORDER && np > 0) {
    const bool pairs_on = c.nonbonded && c.pair != FSL_PAIR_NONE;
    P.nolist = !pairs_on;
    const double cell = std::min(c.lx / P.mnx, std::min(c.ly / P.mny, c.lz / P.mnz));
    const double skin = std::min(0.25 * c.cutoff, 2.0 * cell - c.cutoff);
    const char* env = std::getenv("FLUAMSL_VERLET");
    if (pairs_on && c.pair == FSL_PAIR_SOFT && cell >= c.cutoff && skin >= 0.05 * c.cutoff &&
        !(env && env[0] == '0')) {
      P.verlet = 1;
      P.skin = skin;
      P.vl_cut2 = (c.cutoff + skin) * (c.cutoff + skin);
      P.vl_half2 = 0.25 * skin * skin;
    }
  }
  P.eta = c.shearviscosity;
  P.kT = c.temperature;
  P.dt = c.dt;
  P.extra_mob = c.extra_mobility;
  // src/createCellsStokesLimitGPU.cu:58-61
  P.fact1 = std::sqrt((4. * c.temperature * c.shearviscosity) / (P.dV * c.dt));
  P.fact4 = std::sqrt((2. * c.temperature * c.shearviscosity) / (P.dV * c.dt));
  P.fact2 = std::sqrt(c.temperature * c.extra_mobility * c.dt);
  P.seed = c.seed;
  P.keys = philox_keys(P.seed);
  if (two_d) {
    // src/createCellsQuasi2DGPU.cu:49-79: blob variance by scheme, stencil
    // half-width int(3 a mx / lx) + 1 (at most mx / 2), stochastic prefactor
    const double a = c.radius, pi = 3.1415926535897932385;
    P.q2_var = c.scheme == FSL_SCHEME_QUASI2D ? std::pow(a / std::sqrt(pi), 2)
                                              : std::pow(a * 0.66556976637237890625, 2);
    P.q2_kw = (int)(3.0 * a * c.mx / c.lx) + 1;
    if (P.q2_kw > c.mx / 2) P.q2_kw = c.mx / 2;
    P.q2_fact1 = std::sqrt(1.0 * c.temperature / (c.shearviscosity * c.dt * c.lx * c.ly)) * (double)P.nc;
    P.q2_kc = c.saffman_kc;
    P.q2_lw = c.saffman_width;
    P.q2_shear = c.shear_amp;
    P.q2_rfd = c.use_rfd ? 1 : 0;
    P.q2_pc = c.predictor_corrector ? 1 : 0;
    P.q2_ndrift = c.ndrift;
    P.prec = PREC_F64;  // FP64 throughout, as the reference
  }
  if (incomp) {
    // src/createCellsIncompressibleGPU.cu:60-63
    const double rho = c.density, T = c.temperature, eta = c.shearviscosity, dt = c.dt;
    P.rho = rho;
    P.fact1 = std::sqrt((4. * T * eta * dt) / (P.dV * rho * rho));
    P.fact4 = std::sqrt((2. * T * eta * dt) / (P.dV * rho * rho));
    P.prec = PREC_F64;  // FP64 throughout, as the reference
  }
  P.noise_n = noise_count(P, P.np);
  return FSL_OK;
}

void build_ljtable(const Params& P, double temperature, double cutoff, std::vector<float>& t) {
  const int size = kLjTableSize;
  t.assign(size, 0.0f);
  float sigma = (float)(2.0 * P.lx / (double)P.mx);
  float epsilon = (float)temperature;
  float cutoff2 = (float)(cutoff * cutoff);
  float dr = cutoff2 / (float)size;
  float r = 0.5f * dr;
  for (int i = 0; i < size; ++i) {
    double rr = (double)sqrtf(r);
    float fr = (float)(48. * epsilon * (std::pow(sigma / rr, 12) - 0.5 * std::pow(sigma / rr, 6)) / rr);
    t[i] = fr / sqrtf(r);
    r += dr;
  }
  t[size - 1] = 0.0f;
  t[0] = 0.0f;
}

// ------------------------------------------------------------------ slots --
size_t slot_bytes(const Params& P, int np_cap) { return layout(P, np_cap).total; }

int slot_alloc(Slot& s, const Params& P, int np_cap, cudaStream_t st) {
  slot_free(s);
  const SlotLayout L = layout(P, np_cap);
  char* base = nullptr;
  FSL_TRY(cudaMalloc((void**)&base, L.total));
  s.arena = base;
  s.bytes = L.total;
  s.np_cap = np_cap;
  // on the stream of the uploads that follow: a memset on the legacy default
  // stream is not ordered with a non-blocking stream and could land after them
  cudaError_t e = cudaMemsetAsync(base, 0, L.total, st);
  if (e != cudaSuccess) {
    slot_free(s);
    return cuda_fail(e, "cudaMemset(slot)");
  }
  Rep& r = s.r;
  std::memset(&r, 0, sizeof(r));
  r.P = P;
  r.active = 0;
  r.q = (double*)(base + L.q);
  r.qp = (double*)(base + L.qp);
  r.F = (double*)(base + L.F);
  r.u = (double*)(base + L.u);
  r.qw = (double*)(base + L.qw);
  r.ws = (double*)(base + L.ws);
  r.cell_of = (int*)(base + L.cell_of);
  r.tmp = (int*)(base + L.tmp);
  r.sorted = (int*)(base + L.sorted);
  r.bpp_cnt = (int*)(base + L.bpp_cnt);
  r.bpp_off = (int*)(base + L.bpp_off);
  r.bfp_cnt = (int*)(base + L.bfp_cnt);
  r.bfp_off = (int*)(base + L.bfp_off);
  r.cnt = (int*)(base + L.cnt);
  r.fill = (int*)(base + L.fill);
  r.start = (int*)(base + L.start);
  r.bsum = (int*)(base + L.bsum);
  r.ljtab = (float*)(base + L.ljtab);
  r.noise = (float*)(base + L.noise);
  r.ndiv = (float*)(base + L.ndiv);
  r.stc = P.prec != FSL_PRECISION_FP64 && P.scheme == FSL_SCHEME_MIDPOINT ? (uint4*)(base + L.stc) : nullptr;
  r.grid = (unsigned long long*)(base + L.grid);
  r.spec = (float2*)(base + L.spec);
  r.v = (float*)(base + L.v);
  r.wbuf = (float*)(base + L.wbuf);
  const bool f64 = P.prec == FSL_PRECISION_FP64;
  r.noise64 = f64 ? (double*)(base + L.noise64) : nullptr;
  r.v64 = f64 ? (double*)(base + L.v64) : nullptr;
  r.z64 = f64 ? (double2*)(base + L.z64) : nullptr;
  r.err = (int*)(base + L.err);
  r.t = (uint64_t*)(base + L.t);
  r.q0 = P.observe ? (double*)(base + L.q0) : nullptr;
  r.obs = (double*)(base + L.obs);
  r.obs_part = P.observe ? (double*)(base + L.obs_part) : nullptr;
  r.obs_ticket = (unsigned*)(base + L.obs_ticket);
  const bool two_lists = P.scheme <= FSL_SCHEME_FIRST_ORDER;
  r.start1 = two_lists ? (int*)(base + L.start1) : nullptr;
  r.sorted1 = two_lists ? (int*)(base + L.sorted1) : nullptr;
  r.ws1 = two_lists ? (double*)(base + L.ws1) : nullptr;
  r.vl_cnt = P.verlet ? (int*)(base + L.vl_cnt) : nullptr;
  r.vl_idx = P.verlet ? (int*)(base + L.vl_idx) : nullptr;
  r.qref = P.verlet ? (double*)(base + L.qref) : nullptr;
  r.vl_flag = (uint64_t*)(base + L.vl_flag);
  r.bar = (unsigned*)(base + L.bar);  // zeroed with the slot
  return FSL_OK;
}

void slot_free(Slot& s) {
  if (s.arena) cudaFree(s.arena);
  if (s.bonds) cudaFree(s.bonds);
  s.arena = s.bonds = nullptr;
  s.bytes = 0;
  s.np_cap = 0;
  std::memset(&s.r, 0, sizeof(s.r));
}

int slot_read_observables(const Slot& s, cudaStream_t st, fsl_observables* out) {
  const Rep& r = s.r;
  if (!r.P.observe) return errorf(FSL_E_ARG, "observables are off (fsl_config.observables = 0)");
  double o[kObsSlots];
  FSL_TRY(cudaMemcpyAsync(o, r.obs, sizeof(o), cudaMemcpyDeviceToHost, st));
  FSL_TRY(cudaStreamSynchronize(st));
  std::memset(out, 0, sizeof(*out));
  out->steps = (int64_t)o[0];
  out->msd = o[1];
  out->msd_sum = o[2];
  for (int d = 0; d < 3; ++d) {
    out->displacement[d] = o[3 + d];
    out->force[d] = o[6 + d];
    out->momentum[d] = o[9 + d];
    out->momentum_sum[d] = o[12 + d];
  }
  return FSL_OK;
}

int slot_clear_errors(Slot& s, cudaStream_t st) {
  FSL_TRY(cudaMemsetAsync(s.r.err, 0, sizeof(int) * 4, st));
  launch_reset_lists(s.r, st);
  FSL_TRY(cudaGetLastError());
  return slot_force_lists(s, st);
}

int slot_force_lists(Slot& s, cudaStream_t st) {
  static const uint64_t flags[3] = {0, 0, 1};
  FSL_TRY(cudaMemcpyAsync(s.r.vl_flag, flags, sizeof(flags), cudaMemcpyHostToDevice, st));
  return FSL_OK;
}

int slot_mark_moved(Slot& s, cudaStream_t st) {
  launch_moved_check(s.r, st);
  FSL_TRY(cudaGetLastError());
  return FSL_OK;
}

int slot_request_lists(Slot& s, cudaStream_t st) {
  static const uint64_t two = 2;
  FSL_TRY(cudaMemcpyAsync(s.r.vl_flag + 2, &two, sizeof(two), cudaMemcpyHostToDevice, st));
  return FSL_OK;
}

int slot_reset_observables(Slot& s, cudaStream_t st) {
  Rep& r = s.r;
  if (r.P.observe && r.P.np > 0)
    FSL_TRY(cudaMemcpyAsync(r.q0, r.q, sizeof(double) * 3 * (size_t)r.P.np, cudaMemcpyDeviceToDevice, st));
  FSL_TRY(cudaMemsetAsync(r.obs, 0, sizeof(double) * kObsSlots, st));
  FSL_TRY(cudaMemsetAsync(r.obs_ticket, 0, sizeof(unsigned), st));
  return FSL_OK;
}

int slot_reset(Slot& s, const Params& P, const double* q, const fsl_config& c, cudaStream_t st) {
  if (!s.arena) return errorf(FSL_E_ARG, "slot not allocated");
  if (P.np > s.np_cap) return errorf(FSL_E_ARG, "%d particles exceed the slot's %d", P.np, s.np_cap);
  if (!(class_of(P) == class_of(s.r.P))) return errorf(FSL_E_ARG, "instance is not of the slot's size class");
  if (P.np > 0 && !q) return errorf(FSL_E_ARG, "null positions");
  Rep& r = s.r;
  r.P = P;
  r.P.bonded = 0;
  r.bpp_idx = nullptr;
  r.bpp_k = r.bpp_r0 = nullptr;
  r.bfp_k = r.bfp_r0 = r.bfp_xyz = nullptr;
  const size_t n3p = 3 * (size_t)P.np, cap = (size_t)std::max(s.np_cap, 1);
  if (P.np > 0) {
    FSL_TRY(cudaMemcpyAsync(r.q, q, sizeof(double) * n3p, cudaMemcpyHostToDevice, st));
    FSL_TRY(cudaMemcpyAsync(r.qp, q, sizeof(double) * n3p, cudaMemcpyHostToDevice, st));
  }
  std::vector<float> tab;
  build_ljtable(P, c.temperature, c.cutoff, tab);
  // pageable source: the copy is staged before the call returns
  FSL_TRY(cudaMemcpyAsync(r.ljtab, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice, st));
  FSL_TRY(cudaMemsetAsync(r.F, 0, sizeof(double) * 3 * cap, st));
  FSL_TRY(cudaMemsetAsync(r.bpp_cnt, 0, sizeof(int) * cap, st));
  FSL_TRY(cudaMemsetAsync(r.bpp_off, 0, sizeof(int) * cap, st));
  FSL_TRY(cudaMemsetAsync(r.bfp_cnt, 0, sizeof(int) * cap, st));
  FSL_TRY(cudaMemsetAsync(r.bfp_off, 0, sizeof(int) * cap, st));
  // the step's cell-list builds rely on cleared counters
  FSL_TRY(cudaMemsetAsync(r.cnt, 0, sizeof(int) * (size_t)P.mN, st));
  FSL_TRY(cudaMemsetAsync(r.fill, 0, sizeof(int) * (size_t)P.mN, st));
  FSL_TRY(cudaMemsetAsync(r.grid, 0, sizeof(unsigned long long) * 3 * (size_t)P.nc, st));
  if (P.prec == PREC_F64)
    FSL_TRY(cudaMemsetAsync(r.v64, 0, sizeof(double) * 3 * (size_t)P.nc, st));
  else
    FSL_TRY(cudaMemsetAsync(r.v, 0, sizeof(float) * 3 * (size_t)P.nc, st));
  FSL_TRY(cudaMemsetAsync(r.err, 0, sizeof(int) * 4, st));
  if (r.bar) FSL_TRY(cudaMemsetAsync(r.bar, 0, sizeof(unsigned) * 2, st));
  FSL_TRY(cudaMemsetAsync(r.t, 0, sizeof(uint64_t), st));
  if (int rc = slot_reset_observables(s, st)) return rc;
  if (int rc = slot_force_lists(s, st)) return rc;
  r.active = 1;
  return FSL_OK;
}

int slot_bonds(Slot& s, int64_t nbonds, const int32_t* bi, const int32_t* bj, const double* k,
               const double* r0, int64_t nfixed, const int32_t* fi, const double* fk,
               const double* fr0, const double* fxyz, cudaStream_t st, bool directed) {
  Rep& r = s.r;
  const int np = r.P.np;
  if (nbonds < 0 || nfixed < 0) return errorf(FSL_E_ARG, "negative bond count");
  if (nbonds > 0 && (!bi || !bj || !k || !r0)) return errorf(FSL_E_ARG, "null bond array");
  if (nfixed > 0 && (!fi || !fk || !fr0 || !fxyz)) return errorf(FSL_E_ARG, "null tether array");
  for (int64_t b = 0; b < nbonds; ++b)
    if (bi[b] < 0 || bi[b] >= np || bj[b] < 0 || bj[b] >= np)
      return errorf(FSL_E_ARG, "bond %lld: particle index out of range", (long long)b);
  for (int64_t b = 0; b < nfixed; ++b)
    if (fi[b] < 0 || fi[b] >= np)
      return errorf(FSL_E_ARG, "tether %lld: particle index out of range", (long long)b);
  // both endpoints store each particle-particle bond, in file order; a
  // directed entry (the old bond-file format) is stored by bi only
  std::vector<int> pc(np, 0), po(np, 0), fc(np, 0), fo(np, 0), tmp(np, 0);
  for (int64_t b = 0; b < nbonds; ++b) {
    pc[bi[b]]++;
    if (!directed) pc[bj[b]]++;
  }
  for (int64_t b = 0; b < nfixed; ++b) fc[fi[b]]++;
  for (int i = 1; i < np; ++i) {
    po[i] = po[i - 1] + pc[i - 1];
    fo[i] = fo[i - 1] + fc[i - 1];
  }
  const int64_t nent = directed ? nbonds : 2 * nbonds;  // stored entries
  std::vector<int> idx(nent);
  std::vector<double> kk(nent), rr(nent);
  for (int64_t b = 0; b < nbonds; ++b) {
    int i1 = bi[b], i2 = bj[b];
    int p1 = po[i1] + tmp[i1]++;
    idx[p1] = i2;
    kk[p1] = k[b];
    rr[p1] = r0[b];
    if (directed) continue;
    int p2 = po[i2] + tmp[i2]++;
    idx[p2] = i1;
    kk[p2] = k[b];
    rr[p2] = r0[b];
  }
  std::fill(tmp.begin(), tmp.end(), 0);
  std::vector<double> fkk(nfixed), frr(nfixed), fxx(3 * nfixed);
  for (int64_t b = 0; b < nfixed; ++b) {
    int i1 = fi[b];
    int p = fo[i1] + tmp[i1]++;
    fkk[p] = fk[b];
    frr[p] = fr0[b];
    fxx[3 * p] = fxyz[3 * b];
    fxx[3 * p + 1] = fxyz[3 * b + 1];
    fxx[3 * p + 2] = fxyz[3 * b + 2];
  }
  // one allocation for the tables: idx | k | r0 | fk | fr0 | fxyz
  const size_t nb2 = (size_t)nent, nf = (size_t)nfixed;
  const size_t o_idx = 0, o_k = align_up(sizeof(int) * nb2), o_r0 = o_k + align_up(sizeof(double) * nb2),
               o_fk = o_r0 + align_up(sizeof(double) * nb2), o_fr0 = o_fk + align_up(sizeof(double) * nf),
               o_fx = o_fr0 + align_up(sizeof(double) * nf), total = o_fx + align_up(sizeof(double) * 3 * nf);
  FSL_TRY(cudaStreamSynchronize(st));  // the old tables may still be read
  if (s.bonds) cudaFree(s.bonds);
  s.bonds = nullptr;
  char* base = nullptr;
  FSL_TRY(cudaMalloc((void**)&base, std::max<size_t>(total, kAlign)));
  s.bonds = base;
  r.bpp_idx = (int*)(base + o_idx);
  r.bpp_k = (double*)(base + o_k);
  r.bpp_r0 = (double*)(base + o_r0);
  r.bfp_k = (double*)(base + o_fk);
  r.bfp_r0 = (double*)(base + o_fr0);
  r.bfp_xyz = (double*)(base + o_fx);
  if (np > 0) {
    FSL_TRY(cudaMemcpyAsync(r.bpp_cnt, pc.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st));
    FSL_TRY(cudaMemcpyAsync(r.bpp_off, po.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st));
    FSL_TRY(cudaMemcpyAsync(r.bfp_cnt, fc.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st));
    FSL_TRY(cudaMemcpyAsync(r.bfp_off, fo.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st));
  }
  if (nbonds > 0) {
    FSL_TRY(cudaMemcpyAsync(r.bpp_idx, idx.data(), sizeof(int) * nb2, cudaMemcpyHostToDevice, st));
    FSL_TRY(cudaMemcpyAsync(r.bpp_k, kk.data(), sizeof(double) * nb2, cudaMemcpyHostToDevice, st));
    FSL_TRY(cudaMemcpyAsync(r.bpp_r0, rr.data(), sizeof(double) * nb2, cudaMemcpyHostToDevice, st));
  }
  if (nfixed > 0) {
    FSL_TRY(cudaMemcpyAsync(r.bfp_k, fkk.data(), sizeof(double) * nf, cudaMemcpyHostToDevice, st));
    FSL_TRY(cudaMemcpyAsync(r.bfp_r0, frr.data(), sizeof(double) * nf, cudaMemcpyHostToDevice, st));
    FSL_TRY(cudaMemcpyAsync(r.bfp_xyz, fxx.data(), sizeof(double) * 3 * nf, cudaMemcpyHostToDevice, st));
  }
  // staged copies of host vectors that end here: wait for them
  FSL_TRY(cudaStreamSynchronize(st));
  r.P.bonded = (nbonds + nfixed) > 0;
  return FSL_OK;
}

// ----------------------------------------------------------------- groups --
int group_init(Group& g, const Params& P0) {
  g.key = class_of(P0);
  g.P0 = P0;
  g.fft = fft_plan_create(P0);
  if (!g.fft) return errorf(FSL_E_ARG, "FFT plan creation failed (sizes or shared memory)");
  // lowest priority: the block scheduler fills the SMs with the step's own
  // (latency-bound) kernels first and the noise takes the rest
  int lo = 0, hi = 0;
  FSL_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  FSL_TRY(cudaStreamCreateWithPriority(&g.side, cudaStreamNonBlocking, lo));
  FSL_TRY(cudaEventCreateWithFlags(&g.ev_fork, cudaEventDisableTiming));
  FSL_TRY(cudaEventCreateWithFlags(&g.ev_join, cudaEventDisableTiming));
  FSL_TRY(cudaEventCreateWithFlags(&g.ev_join2, cudaEventDisableTiming));
  for (int i = 0; i < 2; ++i) {
    FSL_TRY(cudaEventCreateWithFlags(&g.ev_w[i], cudaEventDisableTiming));
    FSL_TRY(cudaEventCreateWithFlags(&g.ev_c[i], cudaEventDisableTiming));
  }
  tile_init();
  return FSL_OK;
}

void group_destroy(Group& g) {
  if (g.side) {
    cudaStreamSynchronize(g.side);
    cudaStreamDestroy(g.side);
  }
  if (g.ev_fork) cudaEventDestroy(g.ev_fork);
  if (g.ev_join) cudaEventDestroy(g.ev_join);
  if (g.ev_join2) cudaEventDestroy(g.ev_join2);
  for (int i = 0; i < 2; ++i) {
    if (g.ev_w[i]) cudaEventDestroy(g.ev_w[i]);
    if (g.ev_c[i]) cudaEventDestroy(g.ev_c[i]);
    g.ev_w[i] = g.ev_c[i] = nullptr;
  }
  g.side = nullptr;
  g.ev_fork = g.ev_join = g.ev_join2 = nullptr;
  fft_plan_destroy(g.fft);
  g.fft = nullptr;
  if (g.d_reps) cudaFree(g.d_reps);
  if (g.d_boff) cudaFree(g.d_boff);
  g.d_reps = nullptr;
  g.d_boff = nullptr;
  g.d_cap = 0;
  for (int i = 0; i < Prof::kMax; ++i)
    if (g.prof.ev[i]) cudaEventDestroy(g.prof.ev[i]);
  std::memset(g.prof.ev, 0, sizeof(g.prof.ev));
}

int group_upload(Group& g) {
  const int n = (int)g.slots.size();
  Batch& B = g.B;
  B.nrep = n;
  B.mx = g.P0.mx;
  B.my = g.P0.my;
  B.mz = g.P0.mz;
  B.mxh = g.P0.mxh;
  B.nc = g.P0.nc;
  B.mN = g.P0.mN;
  B.kernel = g.P0.kernel;
  B.prec = g.P0.prec;
  B.max_np = 0;
  B.max_noise_n = 0;
  // FLUAMSL_TILED_SPREAD=1 puts the fixed-point form's spread and W build on
  // the tiled kernel (same bits).  Off by default: at the benchmark's
  // particle density the global-atomic spread plus the W build is faster.
  const char* env = std::getenv("FLUAMSL_TILED_SPREAD");
  B.tiled = env && env[0] == '1' && tile_eligible(g.P0);
  B.has_vl = B.has_cl = 0;
  for (const Slot* s : g.slots) {
    B.max_np = std::max(B.max_np, s->np_cap);
    B.max_noise_n = std::max<uint64_t>(B.max_noise_n, noise_count(g.P0, s->np_cap));
    B.tiled = B.tiled && tile_eligible(s->r.P);  // per instance: the cell sizes
    if (s->r.P.verlet || s->r.P.nolist) B.has_vl = 1;
    else B.has_cl = 1;
  }
  if (n > g.d_cap) {
    if (g.d_reps || g.d_boff) {
      FSL_TRY(cudaStreamSynchronize(g.stream));
      cudaFree(g.d_reps);
      cudaFree(g.d_boff);
      g.d_reps = nullptr;
      g.d_boff = nullptr;
      g.d_cap = 0;
    }
    int cap = std::max(n, 1);
    FSL_TRY(cudaMalloc((void**)&g.d_reps, sizeof(Rep) * cap));
    FSL_TRY(cudaMalloc((void**)&g.d_boff, sizeof(int) * NKIND * (cap + 1)));
    g.d_cap = cap;
    g.dirty = true;
  }
  B.reps = g.d_reps;
  B.boff = g.d_boff;
  if (!g.dirty) return FSL_OK;
  g.h_reps.resize(n);
  for (int i = 0; i < n; ++i) g.h_reps[i] = g.slots[i]->r;
  // first block of every instance per particle launch kind, from the
  // capacities (fixed while the slots are), so the launch shapes stay put
  g.h_boff.assign((size_t)NKIND * (n + 1), 0);
  for (int k = 0; k < NKIND; ++k) {
    int* off = g.h_boff.data() + (size_t)k * (n + 1);
    long acc = 0;
    for (int i = 0; i < n; ++i) {
      off[i] = (int)acc;
      acc += ((long)g.slots[i]->np_cap + kind_ppb(k) - 1) / kind_ppb(k);
    }
    off[n] = (int)acc;
    if (acc > (long)INT_MAX / 2) return errorf(FSL_E_ARG, "batch too large for one launch");
    B.nblk[k] = (int)acc;
  }
  B.one = (n == 1 && g.allow_one) ? &g.h_reps[0] : nullptr;
  if (n > 0) {
    FSL_TRY(cudaMemcpyAsync(g.d_reps, g.h_reps.data(), sizeof(Rep) * n, cudaMemcpyHostToDevice,
                            g.stream));
    FSL_TRY(cudaMemcpyAsync(g.d_boff, g.h_boff.data(), sizeof(int) * g.h_boff.size(),
                            cudaMemcpyHostToDevice, g.stream));
  }
  g.dirty = false;
  return FSL_OK;
}

void group_tuning(const Group& g, fsl_class_tuning* out) {
  std::memset(out, 0, sizeof(*out));
  out->mx = g.key.mx;
  out->my = g.key.my;
  out->mz = g.key.mz;
  out->kernel = g.key.kernel;
  out->precision = g.key.prec;
  out->scheme = g.key.scheme;
  out->n = (int32_t)g.slots.size();
  FftTuning t;
  fft_tuning(g.fft, t);
  out->tuned = t.tuned;
  out->fft_schedule = t.schedule;
  out->z_tile_kx = t.z_kx;
  out->z_tile_ky = t.z_ky;
  out->z_threads = t.z_threads;
  out->z_candidates = t.nz;
  for (int i = 0; i < 8; ++i) out->z_us[i] = t.z_us[i];
  out->schedule_us[0] = t.sched_us[0];
  out->schedule_us[1] = t.sched_us[1];
  out->plane_pb = t.plane_pb;
  out->plane_candidates = t.npc;
  for (int i = 0; i < 4; ++i) out->plane_us[i] = t.plane_us[i];
  const Batch& B = g.B;
  out->list_build = B.max_np == 0 ? -1 : (B.one && B.one->bar) ? 2 : block_lists(B) ? 1 : 0;
  out->list_us[0] = g.lists_us[0];
  out->list_us[1] = g.lists_us[1];
}

// One midpoint step (src/runSchemeStokesLimit.cu:163-275) of every active
// instance of the group.
void group_enqueue_step(Group& g) {
  const Batch& B = g.B;
  cudaStream_t s = g.stream;
  Prof& pr = g.prof;
  pr.used = 0;
  pr.launches = 0;
  if (B.nrep == 0) {
    g.launches = 0;
    return;
  }
  const int pk = B.max_np > 0 ? 1 : 0;
  // the z-pass tile of this size class, timed on its own buffers (first
  // uncaptured step only)
  if (g.key.scheme <= FSL_SCHEME_FIRST_ORDER) fft_autotune(g.fft, B, s);
  // remembers the first stage whose launch was refused, for the message
  auto chk = [&](const char* stage) {
    if (!g.fail_stage && cudaPeekAtLastError() != cudaSuccess) g.fail_stage = stage;
  };
  // fused: the Verlet-list forces are left to the spread that follows at
  // the same positions (launch_spread with forces = true);
  // FLUAMSL_FUSED_FORCES=0 keeps them in their own launch, for comparison
  static const bool fuse_ok = [] {
    const char* e = getenv("FLUAMSL_FUSED_FORCES");
    return !(e && e[0] == '0');
  }();
  // (the FP64 form spreads in its own kernels, which read F)
  const bool fuse = fuse_ok && B.prec != PREC_F64 && !B.tiled;
  auto cells_forces = [&](int which, bool fused) {
    fused = fused && fuse;
    pr.mark(s, "cells");
    // (one cooperative launch for a single instance, one launch of a block
    // per instance for a batch of small instances; on the Verlet path the
    // list kernels return at once unless a rebuild is due)
    if (launch_pair_lists(B, which, s) != cudaSuccess && !g.fail_stage) g.fail_stage = "cells";
    pr.count(!pk ? 0 : ((B.one && B.one->bar) || block_lists(B)) ? 1 : 5 + (B.has_vl ? 1 : 0));
    chk("cells");
    if (!(fused && !B.has_cl)) pr.mark(s, "forces");
    launch_forces(B, which, s, !fused);
    chk("forces");
    pr.count(pk ? (B.has_vl && !fused ? 1 : 0) + (B.has_cl ? 1 : 0) : 0);
  };
  g.fail_stage = nullptr;
  chk("before the step");
  // the noise of step t has no input but the step counter: it runs on the
  // side stream beside the cell list, forces and spread (part 0: the
  // normals and the divergence of stress sample 1, read by the first W
  // build) and beside the first solve (part 1: the divergence of sample 2,
  // read by the second W build), joined before their first readers
  // (profiled steps keep one stream so that the stage intervals stay
  // sequential)
  const bool fork = !pr.on && g.side;
  const bool div = B.prec != PREC_F64 && g.key.scheme <= FSL_SCHEME_FIRST_ORDER;
  const bool two = div && g.key.scheme == FSL_SCHEME_MIDPOINT;
  if (fork) {
    cudaEventRecord(g.ev_fork, s);
    cudaStreamWaitEvent(g.side, g.ev_fork, 0);
    launch_noise(B, g.side, g.key.scheme, 0);
    cudaEventRecord(g.ev_join, g.side);
    if (two) {
      launch_noise(B, g.side, g.key.scheme, 1);
      cudaEventRecord(g.ev_join2, g.side);
    }
  } else {
    pr.mark(s, "noise");
    launch_noise(B, s, g.key.scheme, 0);
    if (two) launch_noise(B, s, g.key.scheme, 1);
  }
  chk("noise");
  pr.count(1 + (div ? 1 : 0) + (two ? 1 : 0));
  // the positions of an input/output step, copied in from pinned host
  // memory beside the noise (which reads no position), then the Verlet-list
  // check of fsl_set_positions
  if (g.io_wait) cudaStreamWaitEvent(s, g.io_wait, 0);
  if (g.io_in && !g.slots.empty()) {
    cudaMemcpyAsync(g.slots[0]->r.q, g.io_in, g.io_bytes, cudaMemcpyHostToDevice, s);
    launch_moved_check(g.slots[0]->r, s);
    chk("positions in");
  }
  auto join_noise = [&]() {
    if (fork) cudaStreamWaitEvent(s, g.ev_join, 0);
  };
  auto join_noise2 = [&]() {
    if (fork && two) cudaStreamWaitEvent(s, g.ev_join2, 0);
  };
  // the field clear after a W build goes to the side stream, where its
  // blocks fill the SMs that the transforms leave idle; the W build then
  // only reads the field
  const bool clear_fork = fork && !B.tiled && B.prec != PREC_F64;
  auto solve = [&](int k, int nsets, double nfac) {
    launch_solve(B, g.fft, nsets, nfac, B.tiled, s, &pr, clear_fork ? g.ev_w[k] : nullptr);
    chk("solve");
    if (!clear_fork) return;
    cudaStreamWaitEvent(g.side, g.ev_w[k], 0);
    launch_field_clear(B, g.side);
    cudaEventRecord(g.ev_c[k], g.side);
    pr.count(1);
  };
  auto join_clear = [&](int k) {
    if (clear_fork) cudaStreamWaitEvent(s, g.ev_c[k], 0);
  };
  auto observe = [&]() {
    if (!g.key.observe) return;
    pr.mark(s, "observe");
    launch_observe(B, s);
    chk("observe");
    pr.count(1);
  };
  if (g.key.scheme == FSL_SCHEME_INCOMPRESSIBLE) {
    // src/runSchemeIncompressible.cu:98-141: two substeps on one noise draw,
    // the advection of the second taken from the prediction
    join_noise();
    pr.mark(s, "inc_substep1");
    launch_inc_w(B, 0, s);
    launch_fft64_3d(B, -1, 0, s);
    launch_inc_fourier(B, 1, s);
    launch_fft64_3d(B, +1, 0, s);
    launch_inc_pred(B, s);
    chk("substep 1");
    pr.mark(s, "inc_substep2");
    launch_inc_w(B, 1, s);
    launch_fft64_3d(B, -1, 0, s);
    launch_inc_fourier(B, 1, s);
    launch_fft64_3d(B, +1, 1, s);
    chk("substep 2");
    pr.count(2 * (1 + 3 + 1 + 3) + 1);
    pr.mark(s, "counter");
    launch_step_counter(B, s);
    chk("counter");
    pr.count(1);
    pr.mark(s, nullptr);
    g.launches = pr.launches;
    return;
  }
  if (g.key.scheme >= FSL_SCHEME_QUASI2D) {
    // src/runSchemeQuasi2D.cu:108-250: 2-D cell list and forces, spread
    // force and thermal drift, Fourier-space mobility and noise, update
    pr.mark(s, "cells");
    launch_cells(B, 0, s, false);
    chk("cells");
    pr.mark(s, "forces");
    launch_q2_forces(B, s);
    chk("forces");
    pr.count(pk ? 6 : 1);
    join_noise();
    launch_q2_field(B, s, &pr);
    chk("spread");
    pr.count(2 + pk);
    launch_q2_solve(B, s, &pr);
    chk("solve");
    pr.count(2 + 1 + 2);
    pr.mark(s, "q2_update");
    launch_q2_update(B, 1, s);
    launch_q2_update(B, 2, s);
    chk("update");
    pr.count(2 * pk);
    pr.mark(s, "counter");
    launch_step_counter(B, s);
    chk("counter");
    pr.count(1);
    pr.mark(s, nullptr);
    g.launches = pr.launches;
    return;
  }
  if (g.key.scheme == FSL_SCHEME_FIRST_ORDER) {
    // src/runSchemeStokesLimitFirstOrder.cu:163-241: f = S(q^n) F^n + RFD
    // drift, one solve with noise factor 1, predictor, forces at q^{n+1/2}
    // only with extraMobility (k_forces returns at once otherwise), corrector
    cells_forces(0, !B.tiled);
    join_noise();
    if (B.tiled) {
      pr.mark(s, "spread_w");
      launch_spread_w(B, 2, 1, 1.0, s);
      chk("spread_w");
      pr.count(1);
    } else {
      pr.mark(s, "spread_rfd");
      launch_spread(B, 2, 1, s, fuse);
      chk("spread_rfd");
      pr.count(pk);
    }
    solve(0, 1, 1.0);
    pr.mark(s, "interp_update");
    launch_interp_update(B, 1, s);
    chk("interp_update");
    pr.count(pk);
    cells_forces(1, false);
    pr.mark(s, "interp_update");
    launch_interp_update(B, 2, s);
    chk("interp_update");
    pr.count(pk);
    observe();
    pr.mark(s, "counter");
    launch_step_counter(B, s);
    chk("counter");
    pr.count(1);
    join_clear(0);
    pr.mark(s, nullptr);
    g.launches = pr.launches;
    return;
  }
  // option 0: F^n, f = S(q^n) F^n; solve 1 with sqrt(2) stress 1.  The
  // spread field is all zeros here: it starts cleared and every W build
  // clears what it reads.  Each spread leaves its nodes and weights in the
  // stencil cache for the interpolation at the same positions (q^n, then
  // q^{n+1/2}) unless the tiled spread, which keeps none, runs.
  const bool stc = !B.tiled;
  // The list build of a batch of small instances: one block per instance or
  // the separate kernels, whichever builds this class's lists faster.  Timed
  // once (first uncaptured step) after the first force evaluation, where a
  // build costs what it costs at most evaluations: the Verlet lists whose
  // rebuild was due are rebuilt by then (the spread that computed the
  // forces has taken the request), the cell lists of the cell-list path and
  // of cell mode rebuild in full.  Both builds give the same lists, and a
  // build at unchanged positions leaves the lists as they are, so the timed
  // builds change no result.
  auto tune_lists = [&]() {
    if (g.lists_tuned || !pk || !block_lists_eligible(B) || block_lists_env() >= 0) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
    g.lists_tuned = true;
    pr.mark(s, "autotune");
    lists_autotune(B, s, g.lists_us);
    g.B.lists_pick = g.lists_us[1] <= g.lists_us[0] ? 1 : 0;
  };
  cells_forces(0, !B.tiled);
  if (B.tiled) {
    join_noise();
    pr.mark(s, "spread_w");
    launch_spread_w(B, 0, 1, 1.41421356237309504880, s);
    chk("spread_w");
    pr.count(1);
  } else {
    pr.mark(s, "spread");
    launch_spread(B, 0, 1, s, fuse, stc);
    chk("spread");
    pr.count(pk);
    join_noise();
  }
  tune_lists();
  solve(0, 1, 1.41421356237309504880);
  // option 1: predictor, F^{n+1/2}, f = S F + RFD; solve 2 with
  // sqrt(1/2) (stress 1 + stress 2)
  pr.mark(s, "interp_update");
  launch_interp_update(B, 1, s, stc);
  chk("interp_update");
  pr.count(pk);
  cells_forces(1, !B.tiled);
  join_clear(0);  // the field is spread into again
  if (B.tiled) {
    join_noise2();
    pr.mark(s, "spread_w_rfd");
    launch_spread_w(B, 1, 2, 0.70710678118654752440, s);
    chk("spread_w_rfd");
    pr.count(1);
  } else {
    pr.mark(s, "spread_rfd");
    launch_spread(B, 1, 1, s, fuse, stc);
    chk("spread_rfd");
    pr.count(pk);
  }
  join_noise2();
  solve(1, 2, 0.70710678118654752440);
  // option 2: corrector
  pr.mark(s, "interp_update");
  launch_interp_update(B, 2, s, stc);
  chk("interp_update");
  pr.count(pk);
  observe();
  pr.mark(s, "counter");
  launch_step_counter(B, s);
  chk("counter");
  pr.count(1);
  join_clear(1);
  pr.mark(s, nullptr);
  g.launches = pr.launches;
}

int group_prof_collect(Group& g) {
  Prof& pr = g.prof;
  if (!pr.on || pr.used < 2) return FSL_OK;
  cudaError_t e = cudaEventSynchronize(pr.ev[pr.used - 1]);
  if (e != cudaSuccess) return errorf(FSL_E_CUDA, "profile sync: %s", cudaGetErrorString(e));
  for (int i = 0; i + 1 < pr.used; ++i) {
    if (!pr.name[i]) continue;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, pr.ev[i], pr.ev[i + 1]);
    auto& a = g.stage_acc[pr.name[i]];
    a.first += 1;
    a.second += ms;
  }
  return FSL_OK;
}

// ------------------------------------------------------------------- exec --
int exec_init(Exec& e, int device) {
  e.device = device;
  FSL_TRY(cudaSetDevice(device));
  // the step's streams take the highest priority, above the noise streams
  int lo = 0, hi = 0;
  FSL_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  FSL_TRY(cudaStreamCreateWithPriority(&e.stream, cudaStreamNonBlocking, hi));
  return FSL_OK;
}

void exec_drop_graph(Exec& e) {
  if (e.gexec) cudaGraphExecDestroy(e.gexec);
  if (e.graph) cudaGraphDestroy(e.graph);
  e.gexec = nullptr;
  e.graph = nullptr;
  e.shape.clear();
}

bool pinned_host(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

void exec_destroy(Exec& e) {
  if (e.stream) cudaStreamSynchronize(e.stream);
  exec_drop_graph(e);
  if (e.io_stream) {
    cudaStreamSynchronize(e.io_stream);
    cudaStreamDestroy(e.io_stream);
    e.io_stream = nullptr;
  }
  if (e.io_fork) cudaEventDestroy(e.io_fork);
  if (e.io_ev) cudaEventDestroy(e.io_ev);
  e.io_fork = e.io_ev = nullptr;
  for (cudaStream_t s : e.side) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  e.side.clear();
  for (cudaEvent_t ev : e.ev) cudaEventDestroy(ev);
  e.ev.clear();
  if (e.stream) cudaStreamDestroy(e.stream);
  e.stream = nullptr;
}

namespace {

int exec_prepare(Exec& e) {
  const size_t ng = e.groups.size();
  while (e.side.size() + 1 < ng) {
    cudaStream_t s;
    int lo = 0, hi = 0;
    FSL_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    FSL_TRY(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, hi));
    e.side.push_back(s);
  }
  while (e.ev.size() < ng + 1) {
    cudaEvent_t ev;
    FSL_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    e.ev.push_back(ev);
  }
  std::vector<long long> shape;
  shape.push_back((long long)(uintptr_t)e.io_key[0]);
  shape.push_back((long long)(uintptr_t)e.io_key[1]);
  if (e.io_in && !e.io_stream) {
    FSL_TRY(cudaStreamCreateWithFlags(&e.io_stream, cudaStreamNonBlocking));
    FSL_TRY(cudaEventCreateWithFlags(&e.io_fork, cudaEventDisableTiming));
    FSL_TRY(cudaEventCreateWithFlags(&e.io_ev, cudaEventDisableTiming));
  }
  for (size_t i = 0; i < ng; ++i) {
    Group& g = *e.groups[i];
    g.stream = i == 0 ? e.stream : e.side[i - 1];
    int rc = group_upload(g);
    if (rc) return rc;
    shape.push_back((long long)(uintptr_t)g.B.reps);
    shape.push_back(g.B.nrep);
    shape.push_back(g.B.max_np);
    shape.push_back((long long)g.B.max_noise_n);
    shape.push_back(g.prof.on ? 1 : 0);
    shape.push_back((long long)(uintptr_t)g.io_in);
    shape.push_back((long long)(uintptr_t)g.io_out);
    for (int k = 0; k < NKIND; ++k) shape.push_back(g.B.nblk[k]);
    // a single instance is a by-value kernel argument: any change to it
    // needs a new capture
    if (g.B.one) {
      long long w[(sizeof(Rep) + 7) / 8] = {};
      std::memcpy(w, g.B.one, sizeof(Rep));
      shape.insert(shape.end(), w, w + (sizeof(Rep) + 7) / 8);
    }
  }
  if (shape != e.shape) {
    exec_drop_graph(e);
    e.shape = shape;
  }
  // the uploads on the side streams must land before the step
  for (size_t i = 1; i < ng; ++i) {
    FSL_TRY(cudaEventRecord(e.ev[i], e.side[i - 1]));
    FSL_TRY(cudaStreamWaitEvent(e.stream, e.ev[i], 0));
  }
  return FSL_OK;
}

void exec_enqueue_groups(Exec& e) {
  const size_t ng = e.groups.size();
  if (ng == 1) {
    Group& g = *e.groups[0];
    group_enqueue_step(g);
    e.launches_per_step = g.launches;
    // the positions after the step of an input/output step
    if (g.io_out && !g.slots.empty())
      cudaMemcpyAsync(g.io_out, g.slots[0]->r.q, g.io_bytes, cudaMemcpyDeviceToHost, e.stream);
    return;
  }
  // fork: every group on its own stream, joined back into the main one
  cudaEventRecord(e.ev[0], e.stream);
  for (size_t i = 1; i < ng; ++i) cudaStreamWaitEvent(e.side[i - 1], e.ev[0], 0);
  int total = 0;
  for (size_t i = 0; i < ng; ++i) {
    group_enqueue_step(*e.groups[i]);
    total += e.groups[i]->launches;
  }
  for (size_t i = 1; i < ng; ++i) {
    cudaEventRecord(e.ev[i], e.side[i - 1]);
    cudaStreamWaitEvent(e.stream, e.ev[i], 0);
  }
  e.launches_per_step = total;
}

void exec_enqueue(Exec& e) {
  const bool io = e.io_in && e.io_stream;
  if (io) {
    // the inputs of an input/output step on the io stream, beside the
    // groups' noise; every group's main branch waits for them
    cudaEventRecord(e.io_fork, e.stream);
    cudaStreamWaitEvent(e.io_stream, e.io_fork, 0);
    e.io_in(e.io_stream);
    cudaEventRecord(e.io_ev, e.io_stream);
    for (Group* g : e.groups) g->io_wait = e.io_ev;
  }
  exec_enqueue_groups(e);
  if (io) {
    for (Group* g : e.groups) g->io_wait = nullptr;
    cudaStreamWaitEvent(e.stream, e.io_ev, 0);
  }
  if (e.io_out) e.io_out(e.stream);
}

}  // namespace

int exec_step(Exec& e, int64_t nsteps) {
  if (nsteps < 0) return errorf(FSL_E_ARG, "negative step count");
  FSL_TRY(cudaSetDevice(e.device));
  if (nsteps == 0) return FSL_OK;
  int rc = exec_prepare(e);
  if (rc) return rc;
  if (e.groups.empty()) return FSL_OK;
  for (int64_t k = 0; k < nsteps; ++k) {
    if (e.use_graph && e.steps > 0) {
      if (!e.gexec) {
        FSL_TRY(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
        exec_enqueue(e);
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(e.stream, &g);
        if (ce != cudaSuccess) return cuda_fail(ce, "graph capture");
        e.graph = g;
        FSL_TRY(cudaGraphInstantiate(&e.gexec, g, 0));
        e.captures++;
      }
      FSL_TRY(cudaGraphLaunch(e.gexec, e.stream));
    } else {
      exec_enqueue(e);
      cudaError_t le = cudaGetLastError();
      if (le != cudaSuccess) {
        for (Group* g : e.groups)
          if (g->fail_stage)
            return errorf(FSL_E_CUDA, "kernel launch (stage %s, cells %d %d %d, kernel %d, %d instances): %s",
                          g->fail_stage, g->key.mx, g->key.my, g->key.mz, g->key.kernel, g->B.nrep,
                          cudaGetErrorString(le));
        return cuda_fail(le, "kernel launch");
      }
    }
    e.steps++;
    for (Group* g : e.groups) {
      rc = group_prof_collect(*g);
      if (rc) return rc;
    }
  }
  return FSL_OK;
}

}  // namespace fsl
