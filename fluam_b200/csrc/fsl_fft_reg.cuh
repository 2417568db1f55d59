// fsl_fft_reg.cuh -- register-resident FFT passes for the compiled cube
// edges (included by fsl_fft.cu only).
//
// A line of N = R * T points is held by T threads: thread t keeps the R
// points x = t + T k (k < R) in registers.  The transform is the two-level
// Cooley-Tukey split N = R x T:
//   1. an R-point DFT over k in registers,          Y_t[a] = sum_k z[t+Tk] W_R^{ak}
//   2. the twiddle W_N^{a t},
//   3. one exchange through shared memory and T-point DFTs over t,
//      X[a + R b] = sum_t W_T^{bt} W_N^{at} Y_t[a],
// so a 1-D transform costs one shared-memory round trip and one barrier
// instead of one per radix stage.  The in-register DFTs are themselves
// mixed-radix (4, 2, 3) splits unrolled at compile time; their twiddles come
// from a constant table read at warp-uniform addresses.

// c_rw[R][j] = exp(-2 pi i j / R) for R <= kMaxRegR (filled by fft_plan_create)
constexpr int kMaxRegR = 44;
__constant__ float2 c_rw[kMaxRegR + 1][kMaxRegR];

template <int R>
__device__ __forceinline__ float2 rw(int j, int dir) {
  float2 w = c_rw[R][j % R];
  if (dir > 0) w.y = -w.y;
  return w;
}

// In-register DFT of size R, natural order in and out:
// V[f] = sum_x v[x] exp(dir 2 pi i f x / R).
template <int R>
struct RDft {
  __device__ __forceinline__ static void run(float2 (&v)[R], int dir) {
    // R = P Q with the small radix P first: x = q + Q p, f = g + P h
    constexpr int P = (R % 4 == 0) ? 4
                      : (R % 2 == 0) ? 2
                      : (R % 3 == 0) ? 3
                      : (R % 5 == 0) ? 5
                      : (R % 7 == 0) ? 7
                                     : 11;
    static_assert(R % P == 0 && R <= kMaxRegR, "register DFT sizes: 2,3,5,7,11-smooth, <= kMaxRegR");
    constexpr int Q = R / P;
    float2 Y[P][Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      float2 u[P];
#pragma unroll
      for (int p = 0; p < P; ++p) u[p] = v[q + Q * p];
      dft<P>(u, dir);
#pragma unroll
      for (int g = 0; g < P; ++g) Y[g][q] = (g * q == 0) ? u[g] : cmul(u[g], rw<R>(g * q, dir));
    }
#pragma unroll
    for (int g = 0; g < P; ++g) {
      RDft<Q>::run(Y[g], dir);
#pragma unroll
      for (int h = 0; h < Q; ++h) v[g + P * h] = Y[g][h];
    }
  }
};
template <>
struct RDft<1> {
  __device__ __forceinline__ static void run(float2 (&)[1], int) {}
};
template <>
struct RDft<2> {
  __device__ __forceinline__ static void run(float2 (&v)[2], int dir) { dft<2>(v, dir); }
};
template <>
struct RDft<3> {
  __device__ __forceinline__ static void run(float2 (&v)[3], int dir) { dft<3>(v, dir); }
};
template <>
struct RDft<4> {
  __device__ __forceinline__ static void run(float2 (&v)[4], int dir) { dft<4>(v, dir); }
};
template <>
struct RDft<5> {
  __device__ __forceinline__ static void run(float2 (&v)[5], int dir) { dft<5>(v, dir); }
};
template <>
struct RDft<7> {
  __device__ __forceinline__ static void run(float2 (&v)[7], int dir) { dft<7>(v, dir); }
};
template <>
struct RDft<11> {
  __device__ __forceinline__ static void run(float2 (&v)[11], int dir) { dft<11>(v, dir); }
};

// Exchange layout of one line: Y_t[a] at [a (T + 1) + t]; the line pitch is
// odd so that neighbouring lines fall on other banks.
template <int R, int T>
struct LineGeom {
  static constexpr int N = R * T;
  static constexpr int XP = T + 1;                    // pitch of one a-row
  static constexpr int EX = (T > 1 ? R * XP : N) | 1;  // exchange floats2 per line
  static constexpr int LS = (EX > N + 1 ? EX : (N + 1)) | 1;  // line pitch (>= N + 1)
  // after the exchange thread t takes RT values of a: a = t RT + j when T
  // divides R, else a = t + T j (j < RT, a < R)
  static constexpr bool EVEN = R % T == 0;
  static constexpr int RT = (R + T - 1) / T;
};

// Exchange layout of the plane kernels' x pass, whose warps hold 32 / T
// lines (row pairs) of T lanes each: line pitch LS, a-row pitch XP and, with
// SW, lane t's value of row a in slot (t + a / RT) mod T of its a-row.
// Chosen so that the exchange write and its read-back each take the
// minimum two wavefronts per warp instruction (8-byte accesses, 16 lanes
// per 128 bytes); with the y-pass geometry the write of the 64 edge took
// eight.  Where and in which slot a value waits changes nothing of the
// arithmetic.
// The inverse's x pass also reads the rows of the half-spectrum plane
// (float2, row pitch PR >= N / 2 + 1) and writes the rows of the real plane
// (float, row pitch PRF >= N); their pitches are chosen the same way.
template <int R, int T>
struct XLineGeom {
  static constexpr int XP = LineGeom<R, T>::XP, LS = LineGeom<R, T>::LS;
  static constexpr bool SW = false;
  static constexpr int PR = R * T / 2 + 1, PRF = R * T + 1;
};
template <>
struct XLineGeom<16, 2> {  // edge 32
  static constexpr int XP = 2, LS = 34;
  static constexpr bool SW = true;
  static constexpr int PR = 17, PRF = 33;
};
template <>
struct XLineGeom<12, 4> {  // edge 48
  static constexpr int XP = 5, LS = 60;
  static constexpr bool SW = false;
  static constexpr int PR = 26, PRF = 50;
};
template <>
struct XLineGeom<16, 4> {  // edge 64
  static constexpr int XP = 4, LS = 68;
  static constexpr bool SW = true;
  static constexpr int PR = 34, PRF = 67;
};
template <>
struct XLineGeom<20, 4> {  // edge 80
  static constexpr int XP = 5, LS = 100;
  static constexpr bool SW = false;
  static constexpr int PR = 42, PRF = 82;
};
template <>
struct XLineGeom<24, 4> {  // edge 96
  static constexpr int XP = 4, LS = 100;
  static constexpr bool SW = true;
  static constexpr int PR = 50, PRF = 98;
};

// slot of lane t's value of a-row a (see XLineGeom)
template <int R, int T, bool SW>
__device__ __forceinline__ int ex_slot(int t, int a) {
  if constexpr (SW) return (t + a / LineGeom<R, T>::RT) % T;
  return t;
}

template <int R, int T>
__device__ __forceinline__ int line_a(int t, int j) {
  return LineGeom<R, T>::EVEN ? t * LineGeom<R, T>::RT + j : t + T * j;
}

// whether slot j of thread t holds a value
template <int R, int T>
__device__ __forceinline__ bool line_has(int t, int j) {
  return LineGeom<R, T>::EVEN || line_a<R, T>(t, j) < R;
}

// Shared memory of one plane in the plane kernels (float2): the line buffer
// of H lines or the row-major half plane of N rows, whichever is larger.
template <int N, int R, int T>
__host__ __device__ constexpr int plane_buf() {
  return (N / 2) * LineGeom<R, T>::LS > N * (N / 2 + 1) ? (N / 2) * LineGeom<R, T>::LS
                                                         : N * (N / 2 + 1);
}

// Steps 1-2 and the exchange write: v holds z[t + T k]; afterwards the line's
// exchange area holds Y_t[a] W_N^{a t}.  tw[i] = exp(-2 pi i i / N) (smem).
// With T == 1 the transform is complete here and v holds X[f] in order.
template <int R, int T, int XP = LineGeom<R, T>::XP, bool SW = false>
__device__ __forceinline__ void line_fft_a(float2 (&v)[R], int t, float2* ex,
                                           const float2* __restrict__ tw, int dir) {
  using G = LineGeom<R, T>;
  static_assert(!SW || G::EVEN, "the slot rotation assumes T divides R");
  RDft<R>::run(v, dir);
  if constexpr (T > 1) {
#pragma unroll
    for (int a = 1; a < R; ++a) {
      float2 w = tw[(a * t) % G::N];
      if (dir > 0) w.y = -w.y;
      v[a] = cmul(v[a], w);
    }
#pragma unroll
    for (int a = 0; a < R; ++a) ex[a * XP + ex_slot<R, T, SW>(t, a)] = v[a];
  }
}

// Step 3 after a barrier: thread t takes its a values (line_a, j < RT) and
// all T values of each; out[j][b] = X[a + R b] (zero where line_has fails).
template <int R, int T, int XP = LineGeom<R, T>::XP, bool SW = false>
__device__ __forceinline__ void line_fft_b(const float2* ex, int t, int dir,
                                           float2 (&out)[LineGeom<R, T>::RT][T]) {
  using G = LineGeom<R, T>;
#pragma unroll
  for (int j = 0; j < G::RT; ++j) {
    const int a = line_a<R, T>(t, j);
    if (!line_has<R, T>(t, j)) {
#pragma unroll
      for (int tt = 0; tt < T; ++tt) out[j][tt] = make_float2(0.f, 0.f);
      continue;
    }
#pragma unroll
    for (int tt = 0; tt < T; ++tt) out[j][tt] = ex[a * XP + ex_slot<R, T, SW>(tt, a)];
    RDft<T>::run(out[j], dir);
  }
}

// frequency of out[j][b] (or of v[j * T + b] when T == 1)
template <int R, int T>
__device__ __forceinline__ int line_freq(int t, int j, int b) {
  return line_a<R, T>(t, j) + R * b;
}

// Real-to-complex transform of whole xy planes (x then y), PB planes per
// block, H * T threads per plane (H = N / 2).  x: the row pair (2p, 2p+1) is
// one complex line; y: columns kx = 1 .. H-1 are complex lines and columns 0
// and H (real after the x transform) travel together as one complex line.
// Output: the half spectrum spec[comp][z][ky][kx], kx <= H.
template <bool ONE, int N, int RR, int T, int PB>
__global__ void __launch_bounds__(PB * (N / 2) * T)
    k_plane_fwd_r(FSL_KARGS, const float2* __restrict__ twn) {
  FSL_REP_AT(blockIdx.z);
  using G = LineGeom<RR, T>;
  constexpr int H = N / 2, TPP = H * T, LS = G::LS;
  extern __shared__ __align__(16) float2 smem[];
  float2* stw = smem;
  const int lp = threadIdx.x / TPP, r = threadIdx.x - lp * TPP;
  float2* buf = smem + N + lp * plane_buf<N, RR, T>();
  for (int i = threadIdx.x; i < N; i += blockDim.x) stw[i] = twn[i];
  const int pl = blockIdx.x * PB + lp;  // comp * mz + z
  const bool live = pl < 3 * P.mz;
  const int comp = live ? pl / P.mz : 0, z = live ? pl - comp * P.mz : 0;
  const float* W = R.wbuf + (size_t)comp * P.nc + (size_t)z * N * N;
  float2 v[RR];
  if constexpr (T == 1) {
    // stage the plane through shared memory so the global reads coalesce
    float* fb = reinterpret_cast<float*>(buf);
    for (int i = r; i < N * N; i += TPP) fb[i + (i / N)] = live ? W[i] : 0.0f;  // row pitch N + 1
    __syncthreads();
    const int p = r;
#pragma unroll
    for (int k = 0; k < RR; ++k) v[k] = make_float2(fb[2 * p * (N + 1) + k], fb[(2 * p + 1) * (N + 1) + k]);
    __syncthreads();
    RDft<RR>::run(v, -1);
#pragma unroll
    for (int f = 0; f < N; ++f) buf[p * LS + f] = v[f];
  } else {
    // The W planes come into the planes' buffers row by row (N floats at
    // pitch PW = N + 4; rows, pitch and buffer starts are multiples of 16
    // bytes) by bulk copies on the block's mbarrier (bounded wait), and the
    // x pass reads them from shared memory: at pitch N + 4 a warp load takes
    // two wavefronts (four at edge 32) where reading the rows from global
    // memory touched eight row segments.
    constexpr int PW = N + 4;
    constexpr unsigned kRowBytes = sizeof(float) * N;
    static_assert(kRowBytes % 16 == 0 && (PW * sizeof(float)) % 16 == 0 && N * PW <= 2 * plane_buf<N, RR, T>() &&
                      plane_buf<N, RR, T>() % 2 == 0 && PB * N * kRowBytes < (1u << 20),
                  "row-wise bulk copies of the W planes");
    __shared__ __align__(8) unsigned long long s_bar;
    if (threadIdx.x == 0) {
      mbar_init(&s_bar, 1);
      mbar_fence_init();
    }
    __syncthreads();
    // blockIdx.x PB < 3 mz, so the block has at least one live plane
    const int nlive = min(PB, 3 * P.mz - (int)blockIdx.x * PB);
    if (threadIdx.x == 0) mbar_arrive_tx(&s_bar, kRowBytes * (unsigned)(N * nlive));
    __syncthreads();
    for (int i = threadIdx.x; i < N * nlive; i += blockDim.x) {
      const int q = i / N, row = i - q * N;
      const int plq = blockIdx.x * PB + q, cq = plq / P.mz, zq = plq - cq * P.mz;
      bulk_load(reinterpret_cast<float*>(smem + N + q * plane_buf<N, RR, T>()) + row * PW,
                R.wbuf + (size_t)cq * P.nc + ((size_t)zq * N + row) * N, kRowBytes, &s_bar);
    }
    bulk_wait(&s_bar, R.err);
    __syncthreads();
    const float* fw = reinterpret_cast<const float*>(buf);  // this thread's plane
    const int p = r / T, t = r - p * T;
#pragma unroll
    for (int k = 0; k < RR; ++k) {
      const int x = t + T * k;
      v[k] = live ? make_float2(fw[(2 * p) * PW + x], fw[(2 * p + 1) * PW + x]) : make_float2(0.f, 0.f);
    }
    __syncthreads();  // the staged plane is overwritten by the exchange
    using XG = XLineGeom<RR, T>;
    static_assert(XG::XP >= T && (RR - 1) * XG::XP + T <= XG::LS && H * XG::LS <= plane_buf<N, RR, T>(),
                  "x-pass exchange fits its line pitch and the plane buffer");
    line_fft_a<RR, T, XG::XP, XG::SW>(v, t, buf + p * XG::LS, stw, -1);
    __syncthreads();
    float2 out[G::RT][T];
    line_fft_b<RR, T, XG::XP, XG::SW>(buf + p * XG::LS, t, -1, out);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < G::RT; ++j)
      if (line_has<RR, T>(t, j))
#pragma unroll
        for (int b = 0; b < T; ++b) buf[p * LS + line_freq<RR, T>(t, j, b)] = out[j][b];
  }
  __syncthreads();
  // y pass: column c, thread t (c fastest, so the stores coalesce)
  const int c = r % H, t = r / H;
#pragma unroll
  for (int k = 0; k < RR; ++k) {
    const int y = t + T * k, p = y >> 1, odd = y & 1;
    if (c == 0) {
      const float2 a = buf[p * LS], b = buf[p * LS + H];
      v[k] = odd ? make_float2(a.y, b.y) : make_float2(a.x, b.x);
    } else {
      const float2 zk = buf[p * LS + c], zm = buf[p * LS + N - c];
      v[k] = odd ? make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x))
                 : make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    }
  }
  __syncthreads();
  float2* out_g = R.spec + ((size_t)comp * P.mz + z) * (size_t)N * (H + 1);
  if constexpr (T == 1) {
    RDft<RR>::run(v, -1);
    if (live) {
      if (c != 0) {
#pragma unroll
        for (int f = 0; f < N; ++f) out_g[(size_t)f * (H + 1) + c] = v[f];
      } else {
#pragma unroll
        for (int f = 0; f < N; ++f) {
          const float2 C = v[f], Cm = v[(N - f) % N];
          out_g[(size_t)f * (H + 1)] = make_float2(0.5f * (C.x + Cm.x), 0.5f * (C.y - Cm.y));
          out_g[(size_t)f * (H + 1) + H] = make_float2(0.5f * (C.y + Cm.y), -0.5f * (C.x - Cm.x));
        }
      }
    }
  } else {
    line_fft_a<RR, T>(v, t, buf + c * LS, stw, -1);
    __syncthreads();
    float2 out[G::RT][T];
    line_fft_b<RR, T>(buf + c * LS, t, -1, out);
    if (live && c != 0) {
#pragma unroll
      for (int j = 0; j < G::RT; ++j)
        if (line_has<RR, T>(t, j))
#pragma unroll
          for (int b = 0; b < T; ++b) out_g[(size_t)line_freq<RR, T>(t, j, b) * (H + 1) + c] = out[j][b];
    }
    __syncthreads();
    // the packed column: C = F0 + i FH, F0 = (C + conj C-)/2, FH = (C - conj C-)/(2i)
    if (c == 0) {
#pragma unroll
      for (int j = 0; j < G::RT; ++j)
        if (line_has<RR, T>(t, j))
#pragma unroll
          for (int b = 0; b < T; ++b) buf[line_freq<RR, T>(t, j, b)] = out[j][b];
    }
    __syncthreads();
    if (c == 0 && live) {
#pragma unroll
      for (int j = 0; j < G::RT; ++j)
        if (line_has<RR, T>(t, j))
#pragma unroll
          for (int b = 0; b < T; ++b) {
          const int f = line_freq<RR, T>(t, j, b);
          const float2 C = out[j][b], Cm = buf[(N - f) % N];
          out_g[(size_t)f * (H + 1)] = make_float2(0.5f * (C.x + Cm.x), 0.5f * (C.y - Cm.y));
          out_g[(size_t)f * (H + 1) + H] = make_float2(0.5f * (C.y + Cm.y), -0.5f * (C.x - Cm.x));
        }
    }
  }
}

// Complex-to-real transform of whole planes, the inverse of k_plane_fwd_r:
// y first (column 0 and H packed again as F0 + i FH), then x with the
// Hermitian completion X[N - f] = conj X[f] of each row; the two real rows of
// a line come out as real and imaginary parts.  Output: v[comp][z][y][x].
template <bool ONE, int N, int RR, int T, int PB>
__global__ void __launch_bounds__(PB * (N / 2) * T)
    k_plane_inv_r(FSL_KARGS, const float2* __restrict__ twn) {
  FSL_REP_AT(blockIdx.z);
  using G = LineGeom<RR, T>;
  // PR: row pitch of the half-spectrum plane, PRF: of the real plane
  constexpr int H = N / 2, TPP = H * T, LS = G::LS, PR = XLineGeom<RR, T>::PR,
                PRF = XLineGeom<RR, T>::PRF;
  static_assert(PR >= H + 1 && N * PR <= plane_buf<N, RR, T>() && PRF >= N &&
                    N * PRF <= 2 * plane_buf<N, RR, T>(),
                "plane rows fit the plane buffer");
  extern __shared__ __align__(16) float2 smem[];
  float2* stw = smem;
  const int lp = threadIdx.x / TPP, r = threadIdx.x - lp * TPP;
  float2* buf = smem + N + lp * plane_buf<N, RR, T>();
  const int pl = blockIdx.x * PB + lp;
  const bool live = pl < 3 * P.mz;
  const int comp = live ? pl / P.mz : 0, z = live ? pl - comp * P.mz : 0;
  // The half-spectrum planes are contiguous (N rows of H + 1, plane pl at
  // pl N (H + 1)): one bulk copy per live plane of the block into the
  // plane's buffer, completed on the block's mbarrier (bounded wait), while
  // the twiddles are staged.  Plane bytes, plane offsets and buffer starts
  // are multiples of 16 bytes.
  constexpr unsigned kPlaneBytes = sizeof(float2) * N * (H + 1);
  static_assert(kPlaneBytes % 16 == 0 && N % 2 == 0 && plane_buf<N, RR, T>() % 2 == 0 &&
                    PB * kPlaneBytes < (1u << 20),
                "bulk copies of whole half-spectrum planes");
  __shared__ __align__(8) unsigned long long s_bar;
  if (threadIdx.x == 0) {
    mbar_init(&s_bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // blockIdx.x PB < 3 mz, so the block has at least one live plane
    const int nlive = min(PB, 3 * P.mz - (int)blockIdx.x * PB);
    mbar_arrive_tx(&s_bar, kPlaneBytes * (unsigned)nlive);
    for (int q = 0; q < nlive; ++q)
      bulk_load(smem + N + q * plane_buf<N, RR, T>(),
                R.spec + (size_t)(blockIdx.x * PB + q) * (size_t)N * (H + 1), kPlaneBytes, &s_bar);
  }
  for (int i = threadIdx.x; i < N; i += blockDim.x) stw[i] = twn[i];
  bulk_wait(&s_bar, R.err);
  __syncthreads();
  const float2* in_s = buf;  // this thread's plane, row pitch H + 1
  // y pass: column c (fastest), thread t
  {
    const int c = r % H, t = r / H;
    float2 v[RR];
#pragma unroll
    for (int k = 0; k < RR; ++k) {
      const int ky = t + T * k;
      if (!live) {
        v[k] = make_float2(0.f, 0.f);
      } else if (c == 0) {
        const float2 f0 = in_s[ky * (H + 1)], fh = in_s[ky * (H + 1) + H];
        v[k] = make_float2(f0.x - fh.y, f0.y + fh.x);  // F0 + i FH
      } else {
        v[k] = in_s[ky * (H + 1) + c];
      }
    }
    __syncthreads();  // the staged plane is overwritten from here on
    if constexpr (T == 1) {
      RDft<RR>::run(v, +1);
      // rows y: X_y[c], or X_y[0] + i X_y[H] for the packed column
#pragma unroll
      for (int y = 0; y < N; ++y) {
        if (c == 0) {
          buf[y * PR] = make_float2(v[y].x, 0.f);
          buf[y * PR + H] = make_float2(v[y].y, 0.f);
        } else {
          buf[y * PR + c] = v[y];
        }
      }
    } else {
      line_fft_a<RR, T>(v, t, buf + c * LS, stw, +1);
      __syncthreads();
      float2 out[G::RT][T];
      line_fft_b<RR, T>(buf + c * LS, t, +1, out);
      __syncthreads();
#pragma unroll
      for (int j = 0; j < G::RT; ++j)
        if (line_has<RR, T>(t, j))
#pragma unroll
          for (int b = 0; b < T; ++b) {
          const int y = line_freq<RR, T>(t, j, b);
          if (c == 0) {
            buf[y * PR] = make_float2(out[j][b].x, 0.f);
            buf[y * PR + H] = make_float2(out[j][b].y, 0.f);
          } else {
            buf[y * PR + c] = out[j][b];
          }
        }
    }
  }
  __syncthreads();
  // x pass: line p = row pair (2p, 2p+1), thread t
  const int p = r / T, t = r - p * T;
  float2 v[RR];
#pragma unroll
  for (int k = 0; k < RR; ++k) {
    const int x = t + T * k;
    float2 e, o;
    if (x <= H) {
      e = buf[(2 * p) * PR + x];
      o = buf[(2 * p + 1) * PR + x];
    } else {
      e = buf[(2 * p) * PR + N - x];
      o = buf[(2 * p + 1) * PR + N - x];
      e.y = -e.y;
      o.y = -o.y;
    }
    v[k] = make_float2(e.x - o.y, e.y + o.x);  // X_2p + i X_2p+1
  }
  __syncthreads();
  float* fb = reinterpret_cast<float*>(buf);  // the real plane, row pitch PRF
  if constexpr (T == 1) {
    RDft<RR>::run(v, +1);
#pragma unroll
    for (int x = 0; x < N; ++x) {
      fb[(2 * p) * PRF + x] = v[x].x;
      fb[(2 * p + 1) * PRF + x] = v[x].y;
    }
  } else {
    using XG = XLineGeom<RR, T>;
    static_assert(XG::XP >= T && (RR - 1) * XG::XP + T <= XG::LS && H * XG::LS <= plane_buf<N, RR, T>(),
                  "x-pass exchange fits its line pitch and the plane buffer");
    line_fft_a<RR, T, XG::XP, XG::SW>(v, t, buf + p * XG::LS, stw, +1);
    __syncthreads();
    float2 out[G::RT][T];
    line_fft_b<RR, T, XG::XP, XG::SW>(buf + p * XG::LS, t, +1, out);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < G::RT; ++j)
      if (line_has<RR, T>(t, j))
#pragma unroll
        for (int b = 0; b < T; ++b) {
        const int x = line_freq<RR, T>(t, j, b);
        fb[(2 * p) * PRF + x] = out[j][b].x;
        fb[(2 * p + 1) * PRF + x] = out[j][b].y;
      }
  }
  __syncthreads();
  if (live) {
    float* out_g = R.v + (size_t)comp * P.nc + (size_t)z * N * N;
    for (int i = r; i < N * N; i += TPP) out_g[i] = fb[(i / N) * PRF + i % N];
  }
}

// z transform, Stokes solve of every mode, inverse z transform, for a tile
// of KX kx values by KY ky values (all three components).  Line
// l = (kyl * 3 + comp) * KX + kxl; thread r = t * nlines + l.  The solve is
// the multiplier of k_zsolve.
template <bool ONE, int MZ, int RR, int T, int KX, int KY>
__global__ void __launch_bounds__(3 * KX * KY * T)
    k_zsolve_r(FSL_KARGS, const float2* __restrict__ twn, const float* __restrict__ sx,
               const float* __restrict__ sy, const float* __restrict__ sz,
               const float2* __restrict__ ex, const float2* __restrict__ ey,
               const float2* __restrict__ ez) {
  FSL_REP_AT(blockIdx.z);
  using G = LineGeom<RR, T>;
  constexpr int NL = 3 * KX * KY, LS = G::LS;
  extern __shared__ float2 smem[];
  float2* stw = smem;
  float2* buf = smem + MZ;
  for (int i = threadIdx.x; i < MZ; i += blockDim.x) stw[i] = twn[i];
  const int my = P.my, mxh = P.mxh;
  const int l = threadIdx.x % NL, t = threadIdx.x / NL;
  const int kxl = l % KX, kyl = (l / KX) / 3, comp = (l / KX) % 3;
  const int kx = blockIdx.x * KX + kxl, ky = blockIdx.y * KY + kyl;
  const bool live = kx < mxh && ky < my;
  const size_t cstride = (size_t)MZ * my * mxh, zstride = (size_t)my * mxh;
  float2* col = R.spec + comp * cstride + (size_t)ky * mxh + kx;
  float2 v[RR];
#pragma unroll
  for (int k = 0; k < RR; ++k) v[k] = live ? col[(size_t)(t + T * k) * zstride] : make_float2(0.f, 0.f);
  __syncthreads();
  float2* lb = buf + l * LS;
  if constexpr (T == 1) {
    RDft<RR>::run(v, -1);
#pragma unroll
    for (int f = 0; f < MZ; ++f) lb[f] = v[f];
  } else {
    line_fft_a<RR, T>(v, t, lb, stw, -1);
    __syncthreads();
    float2 out[G::RT][T];
    line_fft_b<RR, T>(lb, t, -1, out);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < G::RT; ++j)
      if (line_has<RR, T>(t, j))
#pragma unroll
        for (int b = 0; b < T; ++b) lb[line_freq<RR, T>(t, j, b)] = out[j][b];
  }
  __syncthreads();
  // the solve, one thread per (kx, ky, kz) mode
  {
    const float inv_eta = (float)(1.0 / P.eta);
    const float inv_nc = 1.0f / (float)P.nc;
    const float tdx = (float)(2.0 * P.invdx), tdy = (float)(2.0 * P.invdy), tdz = (float)(2.0 * P.invdz);
    // the block size is a multiple of KX * KY, so a thread's (kx, ky) stays
    // the same over its modes and only kz moves: the x and y factors are
    // read once
    static_assert((3 * KX * KY * T) % (KX * KY) == 0, "fixed (kx, ky) per thread");
    const int mxl = threadIdx.x % KX, myl = (threadIdx.x / KX) % KY;
    const int mkx = blockIdx.x * KX + mxl, mky = blockIdx.y * KY + myl;
    const bool mlive = mkx < mxh && mky < my;
    const float2 Ex = mlive ? __ldg(ex + mkx) : make_float2(0.f, 0.f);
    const float2 Ey = mlive ? __ldg(ey + mky) : make_float2(0.f, 0.f);
    // src/initializePrefactorFourierSpace.cu:48-66: g = 2/h sin(pi j/m)
    const float gx = mlive ? tdx * __ldg(sx + mkx) : 0.f, gy = mlive ? tdy * __ldg(sy + mky) : 0.f;
    for (int e = threadIdx.x; e < KX * KY * MZ; e += blockDim.x) {
      const int kz = e / (KX * KY);
      if (!mlive) continue;
      float2* pc[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) pc[a] = buf + ((myl * 3 + a) * KX + mxl) * LS + kz;
      const float2 E[3] = {Ex, Ey, __ldg(ez + kz)};
      const float g[3] = {gx, gy, tdz * __ldg(sz + kz)};
      if (mkx == 0 && mky == 0 && kz == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) *pc[a] = make_float2(0.f, 0.f);
        continue;
      }
      float2 W[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float2 w = *pc[a];
        W[a] = make_float2(w.x * E[a].x + w.y * E[a].y, w.y * E[a].x - w.x * E[a].y);
      }
      const float G2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
      const float invG2 = 1.0f / G2;
      const float2 GW = make_float2(g[0] * W[0].x + g[1] * W[1].x + g[2] * W[2].x,
                                    g[0] * W[0].y + g[1] * W[1].y + g[2] * W[2].y);
      const float fac = inv_eta * invG2 * inv_nc;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float2 V = make_float2((W[a].x - g[a] * GW.x * invG2) * fac, (W[a].y - g[a] * GW.y * invG2) * fac);
        *pc[a] = make_float2(V.x * E[a].x - V.y * E[a].y, V.y * E[a].x + V.x * E[a].y);
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < RR; ++k) v[k] = lb[t + T * k];
  __syncthreads();
  if constexpr (T == 1) {
    RDft<RR>::run(v, +1);
    if (live) {
#pragma unroll
      for (int k = 0; k < RR; ++k) col[(size_t)k * zstride] = v[k];
    }
  } else {
    line_fft_a<RR, T>(v, t, lb, stw, +1);
    __syncthreads();
    float2 out[G::RT][T];
    line_fft_b<RR, T>(lb, t, +1, out);
    if (live) {
#pragma unroll
      for (int j = 0; j < G::RT; ++j)
        if (line_has<RR, T>(t, j))
#pragma unroll
          for (int b = 0; b < T; ++b) col[(size_t)line_freq<RR, T>(t, j, b) * zstride] = out[j][b];
    }
  }
}

// ------------------------------------------------------ warp-local lines ---
// Helpers of the passes whose lines are held by T consecutive lanes of one
// warp (T divides 32, fsl_fft_lines.cuh).

// lanes of this thread's line within its warp
template <int T>
__device__ __forceinline__ unsigned line_mask() {
  if constexpr (T >= 32) return 0xffffffffu;
  else return ((1u << T) - 1u) << ((threadIdx.x & 31) & ~(T - 1));
}

// Stores of one real row segment: the RT consecutive (EVEN layout) values
// out[0..RT)[b] of component sel (0: .x, 1: .y) at x0.
template <int RT, int T>
__device__ __forceinline__ void store_row_run(float* dst, const float2 (&out)[RT][T], int b, int sel) {
  float s[RT];
#pragma unroll
  for (int j = 0; j < RT; ++j) s[j] = sel ? out[j][b].y : out[j][b].x;
  if constexpr (RT == 2) {
    *reinterpret_cast<float2*>(dst) = make_float2(s[0], s[1]);
  } else if constexpr (RT == 4) {
    *reinterpret_cast<float4*>(dst) = make_float4(s[0], s[1], s[2], s[3]);
  } else {
#pragma unroll
    for (int j = 0; j < RT; ++j) dst[j] = s[j];
  }
}
