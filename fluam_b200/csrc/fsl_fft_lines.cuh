// fsl_fft_lines.cuh -- the register-resident transform as five passes of
// warp tasks (included by fsl_fft.cu after fsl_fft_reg.cuh).
//
// The plane kernels of fsl_fft_reg.cuh give a whole xy plane to one block,
// so a 128^3 grid is 384 blocks: 1.3 waves at two blocks per SM, with the
// second wave mostly empty.  Here every pass is split into tasks of one warp
// (32 / T lines of N points, T lanes per line, the lines of a warp
// independent of the other warps), so blocks are short and the last wave
// costs one task:
//   k_fft_xf   x forward of W: row pairs (2p, 2p+1) as one complex line,
//              unpacked into the two half-spectrum rows X[y][kx], kx <= N/2;
//   k_fft_y    y transform of the columns kx = 1 .. N/2 - 1 of every plane,
//              in place; the real columns 0 and N/2 travel together as one
//              complex line (F0 + i FH), as in the plane kernels;
//   k_zsolve_r z forward, Stokes multiplier, z inverse (fsl_fft_reg.cuh);
//   k_fft_y    y inverse;
//   k_fft_xi   x inverse with the Hermitian completion of each row.
// Every line takes the arithmetic of the plane kernels (same split, same
// twiddles, same packing), so both schedules give the same bits and the
// autotuner may pick either per size class.

constexpr int kLineWarps = 8;  // warps per block of the line passes

template <int N>
__device__ __forceinline__ void stage_twiddles(float2* stw, const float2* __restrict__ twn) {
  for (int i = threadIdx.x; i < N; i += blockDim.x) stw[i] = twn[i];
  __syncthreads();
}

// line of this lane: task line L of the launch, lane t of the line; the
// line's exchange area lb (LS float2 per line after the twiddle table)
template <int RR, int T, int N>
__device__ __forceinline__ long line_of(float2* smem, int& t, float2*& lb) {
  constexpr int LW = 32 / T;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int l = lane / T;
  t = lane - l * T;
  lb = smem + N + (warp * LW + l) * LineGeom<RR, T>::LS;
  return ((long)blockIdx.x * kLineWarps + warp) * LW + l;
}

// x forward: the row pair p of plane (comp, z) of W -> half-spectrum rows
// 2p and 2p+1 of spec (row pitch N/2 + 1).  Lines: 3 mz N/2.
template <bool ONE, int N, int RR, int T>
__global__ void __launch_bounds__(kLineWarps * 32) k_fft_xf(FSL_KARGS, const float2* __restrict__ twn) {
  static_assert(32 % T == 0 && T > 1, "warp-local lines");
  FSL_REP_AT(blockIdx.z);
  using G = LineGeom<RR, T>;
  constexpr int H = N / 2;
  extern __shared__ float2 smem[];
  stage_twiddles<N>(smem, twn);
  int t;
  float2* lb;
  const long L = line_of<RR, T, N>(smem, t, lb);
  const bool live = L < 3L * P.mz * H;
  const int plane = live ? (int)(L / H) : 0, p = live ? (int)(L - (long)plane * H) : 0;  // plane = comp mz + z
  const float* row0 = R.wbuf + (size_t)plane * N * N + (size_t)(2 * p) * N;
  const float* row1 = row0 + N;
  float2 v[RR];
#pragma unroll
  for (int k = 0; k < RR; ++k) {
    const int x = t + T * k;
    v[k] = live ? make_float2(row0[x], row1[x]) : make_float2(0.f, 0.f);
  }
  line_fft_a<RR, T>(v, t, lb, smem, -1);
  __syncwarp();
  float2 out[G::RT][T];
  line_fft_b<RR, T>(lb, t, -1, out);
  __syncwarp();
#pragma unroll
  for (int j = 0; j < G::RT; ++j)
    if (line_has<RR, T>(t, j))
#pragma unroll
      for (int b = 0; b < T; ++b) lb[line_freq<RR, T>(t, j, b)] = out[j][b];
  __syncwarp();
  if (!live) return;
  // Z = X_2p + i X_2p+1: X_2p[f] = (Z[f] + conj Z[N-f]) / 2,
  // X_2p+1[f] = (Z[f] - conj Z[N-f]) / (2i)
  float2* o0 = R.spec + ((size_t)plane * N + 2 * p) * (H + 1);
  float2* o1 = o0 + (H + 1);
  for (int f = t; f <= H; f += T) {
    const float2 zk = lb[f], zm = lb[f == 0 ? 0 : N - f];
    o0[f] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    o1[f] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
  }
}

// y transform (DIR -1 forward, +1 inverse) of column kx of plane (comp, z),
// in place in spec; line kx = 0 carries the real columns 0 and N/2.
// Lines: 3 mz N/2.
template <bool ONE, int N, int RR, int T, int DIR>
__global__ void __launch_bounds__(kLineWarps * 32) k_fft_y(FSL_KARGS, const float2* __restrict__ twn) {
  static_assert(32 % T == 0 && T > 1, "warp-local lines");
  FSL_REP_AT(blockIdx.z);
  using G = LineGeom<RR, T>;
  constexpr int H = N / 2, PR = H + 1;
  extern __shared__ float2 smem[];
  stage_twiddles<N>(smem, twn);
  int t;
  float2* lb;
  const long L = line_of<RR, T, N>(smem, t, lb);
  const bool live = L < 3L * P.mz * H;
  const int plane = live ? (int)(L / H) : 0, c = live ? (int)(L - (long)plane * H) : 1;
  float2* col = R.spec + (size_t)plane * N * PR + c;
  float2 v[RR];
#pragma unroll
  for (int k = 0; k < RR; ++k) {
    const int y = t + T * k;
    if (!live) {
      v[k] = make_float2(0.f, 0.f);
    } else if (c != 0) {
      v[k] = col[(size_t)y * PR];
    } else if (DIR < 0) {
      // the real columns 0 and H of the x transform as one complex line
      v[k] = make_float2(col[(size_t)y * PR].x, col[(size_t)y * PR + H].x);
    } else {
      const float2 f0 = col[(size_t)y * PR], fh = col[(size_t)y * PR + H];
      v[k] = make_float2(f0.x - fh.y, f0.y + fh.x);  // F0 + i FH
    }
  }
  line_fft_a<RR, T>(v, t, lb, smem, DIR);
  __syncwarp();
  float2 out[G::RT][T];
  line_fft_b<RR, T>(lb, t, DIR, out);
  if (c != 0) {
    if (live) {
#pragma unroll
      for (int j = 0; j < G::RT; ++j)
        if (line_has<RR, T>(t, j))
#pragma unroll
          for (int b = 0; b < T; ++b) col[(size_t)line_freq<RR, T>(t, j, b) * PR] = out[j][b];
    }
  } else if (DIR > 0) {
    // the two real columns after the inverse: real and imaginary parts
#pragma unroll
    for (int j = 0; j < G::RT; ++j)
      if (line_has<RR, T>(t, j))
#pragma unroll
        for (int b = 0; b < T; ++b) {
          const size_t y = (size_t)line_freq<RR, T>(t, j, b);
          col[y * PR] = make_float2(out[j][b].x, 0.f);
          col[y * PR + H] = make_float2(out[j][b].y, 0.f);
        }
  } else {
    // forward: C = F0 + i FH, F0 = (C + conj C-)/2, FH = (C - conj C-)/(2i)
    const unsigned lm = line_mask<T>();
    __syncwarp(lm);
#pragma unroll
    for (int j = 0; j < G::RT; ++j)
      if (line_has<RR, T>(t, j))
#pragma unroll
        for (int b = 0; b < T; ++b) lb[line_freq<RR, T>(t, j, b)] = out[j][b];
    __syncwarp(lm);
#pragma unroll
    for (int j = 0; j < G::RT; ++j)
      if (line_has<RR, T>(t, j))
#pragma unroll
        for (int b = 0; b < T; ++b) {
          const int f = line_freq<RR, T>(t, j, b);
          const float2 C = out[j][b], Cm = lb[(N - f) % N];
          col[(size_t)f * PR] = make_float2(0.5f * (C.x + Cm.x), 0.5f * (C.y - Cm.y));
          col[(size_t)f * PR + H] = make_float2(0.5f * (C.y + Cm.y), -0.5f * (C.x - Cm.x));
        }
  }
}

// x inverse: half-spectrum rows 2p and 2p+1 of plane (comp, z), completed
// by X[N - x] = conj X[x], as the line X_2p + i X_2p+1; the real and
// imaginary parts are the rows 2p and 2p+1 of v.  Lines: 3 mz N/2.
template <bool ONE, int N, int RR, int T>
__global__ void __launch_bounds__(kLineWarps * 32) k_fft_xi(FSL_KARGS, const float2* __restrict__ twn) {
  static_assert(32 % T == 0 && T > 1, "warp-local lines");
  FSL_REP_AT(blockIdx.z);
  using G = LineGeom<RR, T>;
  constexpr int H = N / 2;
  extern __shared__ float2 smem[];
  stage_twiddles<N>(smem, twn);
  int t;
  float2* lb;
  const long L = line_of<RR, T, N>(smem, t, lb);
  const bool live = L < 3L * P.mz * H;
  const int plane = live ? (int)(L / H) : 0, p = live ? (int)(L - (long)plane * H) : 0;
  const float2* i0 = R.spec + ((size_t)plane * N + 2 * p) * (H + 1);
  const float2* i1 = i0 + (H + 1);
  float2 v[RR];
#pragma unroll
  for (int k = 0; k < RR; ++k) {
    const int x = t + T * k;
    float2 e, o;
    if (!live) {
      e = o = make_float2(0.f, 0.f);
    } else if (x <= H) {
      e = i0[x];
      o = i1[x];
    } else {
      e = i0[N - x];
      o = i1[N - x];
      e.y = -e.y;
      o.y = -o.y;
    }
    v[k] = make_float2(e.x - o.y, e.y + o.x);  // X_2p + i X_2p+1
  }
  line_fft_a<RR, T>(v, t, lb, smem, +1);
  __syncwarp();
  float2 out[G::RT][T];
  line_fft_b<RR, T>(lb, t, +1, out);
  if (!live) return;
  float* row0 = R.v + (size_t)plane * N * N + (size_t)(2 * p) * N;
  float* row1 = row0 + N;
  if constexpr (G::EVEN) {
    // lane t holds x = t RT + j + RR b, j < RT: runs of RT consecutive values
#pragma unroll
    for (int b = 0; b < T; ++b) {
      const int x0 = t * G::RT + RR * b;
      store_row_run<G::RT, T>(row0 + x0, out, b, 0);
      store_row_run<G::RT, T>(row1 + x0, out, b, 1);
    }
  } else {
#pragma unroll
    for (int j = 0; j < G::RT; ++j)
      if (line_has<RR, T>(t, j))
#pragma unroll
        for (int b = 0; b < T; ++b) {
          const int x = line_freq<RR, T>(t, j, b);
          row0[x] = out[j][b].x;
          row1[x] = out[j][b].y;
        }
  }
}
