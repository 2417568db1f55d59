// fsl_fft_v.cuh -- the plane transforms of the 128-point edge with a
// conflict-free shared-memory layout (included by fsl_fft.cu after
// fsl_fft_reg.cuh).
//
// Same arithmetic as k_plane_fwd_r / k_plane_inv_r<N = 128, R = 16, T = 8>
// (the 16 x 8 split, the same twiddle values in the same order), so the two
// give the same bits; what changes is where the values sit in shared memory
// and how wide the accesses are:
//   * exchange of one line: Y_t[a] at t * kVX + a (kVX = 18), so a lane
//     writes its sixteen Y_t[a] as eight 16-byte pairs and reads the pairs
//     (a, a + 1) of every t as eight 16-byte loads; eight lanes of one line
//     (x pass) or of eight lines (y pass, line pitch kVL with kVL / 2 odd)
//     fall on eight distinct 16-byte bank groups;
//   * the twiddles W_N^{a t} of lane t as the same pairs (table kVT);
//   * the real plane in rows of kVR floats (kVR = 8 mod 32), read one float
//     per lane without conflicts, and written as 16-byte rows;
//   * x-pass lines are private to their eight lanes (one quarter warp), so
//     the x exchange needs a warp barrier, not a block barrier;
//   * the inverse's input, the contiguous half-spectrum plane, comes into
//     shared memory by one bulk copy (fsl_bulk.cuh).

constexpr int kVX = 18;   // exchange row of one t (float2)
constexpr int kVL = 146;  // line pitch (float2); kVL / 2 odd
constexpr int kVR = 136;  // real plane row pitch (floats), 544 bytes
constexpr int kVH = 68;   // half-spectrum row pitch in the inverse (float2), 4 mod 8
constexpr int kVT = 8 * kVX;  // twiddle table (float2)

// shared memory of the two kernels (float2): the twiddle table and 64 lines
constexpr int kVSmem = kVT + 64 * kVL;

// twiddle table: twt[t kVX + a] = W_128^{a t} (a < 16), from tw[i] = W^i
__device__ __forceinline__ void v_twiddles(float2* twt, const float2* __restrict__ tw) {
  for (int i = threadIdx.x; i < kVT; i += blockDim.x) {
    const int t = i / kVX, a = i - t * kVX;
    twt[i] = a < 16 ? tw[(a * t) & 127] : make_float2(0.f, 0.f);
  }
}

// Steps 1-2 (line_fft_a): the 16-point DFT of v, the twiddles of lane t,
// the exchange write to the line's area lb.
__device__ __forceinline__ void v_line_a(float2 (&v)[16], int t, float2* lb, const float2* twt, int dir) {
  RDft<16>::run(v, dir);
  const float4* tw4 = reinterpret_cast<const float4*>(twt + t * kVX);
#pragma unroll
  for (int a = 0; a < 16; a += 2) {
    const float4 w2 = tw4[a >> 1];
    float2 w0 = make_float2(w2.x, w2.y), w1 = make_float2(w2.z, w2.w);
    if (dir > 0) {
      w0.y = -w0.y;
      w1.y = -w1.y;
    }
    if (a > 0) v[a] = cmul(v[a], w0);
    v[a + 1] = cmul(v[a + 1], w1);
  }
  float4* ex = reinterpret_cast<float4*>(lb + t * kVX);
#pragma unroll
  for (int a = 0; a < 16; a += 2) ex[a >> 1] = make_float4(v[a].x, v[a].y, v[a + 1].x, v[a + 1].y);
}

// Step 3 (line_fft_b): lane t takes a = 2t + j (j = 0, 1) of every row tt;
// out[j][b] = X[2t + j + 16 b].
__device__ __forceinline__ void v_line_b(const float2* lb, int t, int dir, float2 (&out)[2][8]) {
#pragma unroll
  for (int tt = 0; tt < 8; ++tt) {
    const float4 y = *reinterpret_cast<const float4*>(lb + tt * kVX + 2 * t);
    out[0][tt] = make_float2(y.x, y.y);
    out[1][tt] = make_float2(y.z, y.w);
  }
  RDft<8>::run(out[0], dir);
  RDft<8>::run(out[1], dir);
}

// Forward: W plane (comp, z) -> half spectrum, as k_plane_fwd_r<128,16,8,1>.
template <bool ONE>
__global__ void __launch_bounds__(512) k_plane_fwd_v(FSL_KARGS, const float2* __restrict__ twn) {
  FSL_REP_AT(blockIdx.z);
  constexpr int N = 128, H = 64;
  extern __shared__ __align__(16) float2 smem[];
  float2* twt = smem;
  float2* buf = smem + kVT;
  const int r = threadIdx.x;
  const int pl = blockIdx.x;
  const bool live = pl < 3 * P.mz;
  const int comp = live ? pl / P.mz : 0, z = live ? pl - comp * P.mz : 0;
  v_twiddles(twt, twn);
  // the real plane, 16-byte loads into rows of kVR floats (ordinary loads:
  // measured faster here than bulk row copies or per-thread async copies)
  float* fb = reinterpret_cast<float*>(buf);
  {
    const float4* W4 = reinterpret_cast<const float4*>(R.wbuf + (size_t)comp * P.nc + (size_t)z * N * N);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int i = r + 512 * j, row = i >> 5, x4 = i & 31;
      const float4 w = live ? W4[i] : make_float4(0.f, 0.f, 0.f, 0.f);
      *reinterpret_cast<float4*>(fb + row * kVR + 4 * x4) = w;
    }
  }
  __syncthreads();
  // x pass: line p = rows (2p, 2p+1) as one complex line, lane t
  {
    const int p = r >> 3, t = r & 7;
    float2 v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int x = t + 8 * k;
      v[k] = make_float2(fb[(2 * p) * kVR + x], fb[(2 * p + 1) * kVR + x]);
    }
    __syncthreads();  // the plane's rows are overwritten by the lines
    float2* lb = buf + p * kVL;
    v_line_a(v, t, lb, twt, -1);
    __syncwarp();
    float2 out[2][8];
    v_line_b(lb, t, -1, out);
    __syncwarp();
    // Z[f], f = 2t + j + 16 b, in order: the pairs j = 0, 1 as 16 bytes
#pragma unroll
    for (int b = 0; b < 8; ++b)
      *reinterpret_cast<float4*>(lb + 2 * t + 16 * b) =
          make_float4(out[0][b].x, out[0][b].y, out[1][b].x, out[1][b].y);
  }
  __syncthreads();
  // y pass: column c (fastest), lane t
  const int c = r & (H - 1), t = r >> 6;
  float2 v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int y = t + 8 * k, p = y >> 1, odd = y & 1;
    if (c == 0) {
      const float2 a = buf[p * kVL], b = buf[p * kVL + H];
      v[k] = odd ? make_float2(a.y, b.y) : make_float2(a.x, b.x);
    } else {
      const float2 zk = buf[p * kVL + c], zm = buf[p * kVL + N - c];
      v[k] = odd ? make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x))
                 : make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    }
  }
  __syncthreads();
  float2* out_g = R.spec + ((size_t)comp * P.mz + z) * (size_t)N * (H + 1);
  float2* lb = buf + c * kVL;
  v_line_a(v, t, lb, twt, -1);
  __syncthreads();
  float2 out[2][8];
  v_line_b(lb, t, -1, out);
  if (live && c != 0) {
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int b = 0; b < 8; ++b) out_g[(size_t)(2 * t + j + 16 * b) * (H + 1) + c] = out[j][b];
  }
  __syncthreads();
  // the packed column: C = F0 + i FH, F0 = (C + conj C-)/2, FH = (C - conj C-)/(2i)
  if (c == 0) {
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int b = 0; b < 8; ++b) buf[2 * t + j + 16 * b] = out[j][b];
  }
  __syncthreads();
  if (c == 0 && live) {
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int f = 2 * t + j + 16 * b;
        const float2 C = out[j][b], Cm = buf[(N - f) & (N - 1)];
        out_g[(size_t)f * (H + 1)] = make_float2(0.5f * (C.x + Cm.x), 0.5f * (C.y - Cm.y));
        out_g[(size_t)f * (H + 1) + H] = make_float2(0.5f * (C.y + Cm.y), -0.5f * (C.x - Cm.x));
      }
  }
}

// Inverse: half spectrum -> v plane (comp, z), as k_plane_inv_r<128,16,8,1>.
template <bool ONE>
__global__ void __launch_bounds__(512) k_plane_inv_v(FSL_KARGS, const float2* __restrict__ twn) {
  FSL_REP_AT(blockIdx.z);
  constexpr int N = 128, H = 64;
  extern __shared__ __align__(16) float2 smem[];
  float2* twt = smem;
  float2* buf = smem + kVT;
  const int r = threadIdx.x;
  const int pl = blockIdx.x;
  const bool live = pl < 3 * P.mz;
  const int comp = live ? pl / P.mz : 0, z = live ? pl - comp * P.mz : 0;
  // the half-spectrum plane is contiguous (N rows of H + 1): one bulk copy
  // into shared memory while the block stages the twiddles
  const float2* in_g = R.spec + ((size_t)comp * P.mz + z) * (size_t)N * (H + 1);
  constexpr unsigned kPlaneBytes = N * (H + 1) * sizeof(float2);
  static_assert(kPlaneBytes % 16 == 0 && N * (H + 1) <= 64 * kVL, "plane copy");
  __shared__ __align__(8) unsigned long long s_bar;
  if (r == 0) {
    mbar_init(&s_bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (r == 0 && live) {
    mbar_arrive_tx(&s_bar, kPlaneBytes);
    bulk_load(buf, in_g, kPlaneBytes, &s_bar);
  }
  v_twiddles(twt, twn);
  if (live) bulk_wait(&s_bar, R.err);
  __syncthreads();
  // y pass: column c (fastest), lane t; rows of the result at pitch kVH
  {
    const int c = r & (H - 1), t = r >> 6;
    float2 v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int ky = t + 8 * k;
      if (!live) {
        v[k] = make_float2(0.f, 0.f);
      } else if (c == 0) {
        const float2 f0 = buf[ky * (H + 1)], fh = buf[ky * (H + 1) + H];
        v[k] = make_float2(f0.x - fh.y, f0.y + fh.x);  // F0 + i FH
      } else {
        v[k] = buf[ky * (H + 1) + c];
      }
    }
    __syncthreads();  // the plane is overwritten by the lines
    float2* lb = buf + c * kVL;
    v_line_a(v, t, lb, twt, +1);
    __syncthreads();
    float2 out[2][8];
    v_line_b(lb, t, +1, out);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int y = 2 * t + j + 16 * b;
        if (c == 0) {
          buf[y * kVH] = make_float2(out[j][b].x, 0.f);
          buf[y * kVH + H] = make_float2(out[j][b].y, 0.f);
        } else {
          buf[y * kVH + c] = out[j][b];
        }
      }
  }
  __syncthreads();
  // x pass: line p = row pair (2p, 2p+1) with the Hermitian completion
  const int p = r >> 3, t = r & 7;
  float2 v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int x = t + 8 * k;
    float2 e, o;
    if (x <= H) {
      e = buf[(2 * p) * kVH + x];
      o = buf[(2 * p + 1) * kVH + x];
    } else {
      e = buf[(2 * p) * kVH + N - x];
      o = buf[(2 * p + 1) * kVH + N - x];
      e.y = -e.y;
      o.y = -o.y;
    }
    v[k] = make_float2(e.x - o.y, e.y + o.x);  // X_2p + i X_2p+1
  }
  __syncthreads();
  float2* lb = buf + p * kVL;
  v_line_a(v, t, lb, twt, +1);
  __syncwarp();
  float2 out[2][8];
  v_line_b(lb, t, +1, out);
  __syncthreads();  // the real plane overwrites other lines' areas
  float* fb = reinterpret_cast<float*>(buf);
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const int x = 2 * t + 16 * b;
    *reinterpret_cast<float2*>(fb + (2 * p) * kVR + x) = make_float2(out[0][b].x, out[1][b].x);
    *reinterpret_cast<float2*>(fb + (2 * p + 1) * kVR + x) = make_float2(out[0][b].y, out[1][b].y);
  }
  __syncthreads();
  if (live) {
    float4* out_g = reinterpret_cast<float4*>(R.v + (size_t)comp * P.nc + (size_t)z * N * N);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int i = r + 512 * j, row = i >> 5, x4 = i & 31;
      out_g[i] = *reinterpret_cast<const float4*>(fb + row * kVR + 4 * x4);
    }
  }
}
