// shim_impl.cpp -- out-of-line parts of cuda_host_shim.h.  TEST INFRASTRUCTURE.
#include <complex>
#include <map>
#include <vector>

#include "fsl_oracle.h"

dim3 blockIdx, blockDim, threadIdx, gridDim;

void shim_bad_fetch(const char* what, long i, long n) {
  fprintf(stderr, "reference host build: %s index %ld outside [0, %ld)\n", what, i, n);
  abort();
}

// ---------------------------------------------------------------- cuFFT ---
namespace {
struct Plan {
  int n0, n1, n2;  // n2 varies fastest (cufftPlan3d argument order)
};
std::map<int, Plan> g_plans;
int g_next_plan = 1;

// direct DFT of one line, X_k = sum_j x_j exp(sign 2 pi i j k / n)
void dft_line(std::complex<double>* d, long stride, int n, int sign,
              std::vector<std::complex<double>>& tmp, const std::vector<std::complex<double>>& w) {
  for (int k = 0; k < n; ++k) {
    std::complex<double> acc(0.0, 0.0);
    for (int j = 0; j < n; ++j) acc += d[(long)j * stride] * w[((long)j * k) % n];
    tmp[k] = acc;
  }
  for (int k = 0; k < n; ++k) d[(long)k * stride] = tmp[k];
  (void)sign;
}

std::vector<std::complex<double>> twiddles(int n, int sign) {
  std::vector<std::complex<double>> w(n);
  for (int t = 0; t < n; ++t) {
    double a = 2.0 * M_PI * (double)t / (double)n;
    w[t] = std::complex<double>(std::cos(a), sign * std::sin(a));
  }
  return w;
}
}  // namespace

cufftResult cufftPlan3d(cufftHandle* plan, int nx, int ny, int nz, cufftType) {
  *plan = g_next_plan++;
  g_plans[*plan] = Plan{nx, ny, nz};
  return CUFFT_SUCCESS;
}

cufftResult cufftPlan2d(cufftHandle* plan, int nx, int ny, cufftType) {
  *plan = g_next_plan++;
  g_plans[*plan] = Plan{1, nx, ny};
  return CUFFT_SUCCESS;
}

cufftResult cufftExecZ2Z(cufftHandle plan, cufftDoubleComplex* in, cufftDoubleComplex* out,
                         int direction) {
  const Plan& p = g_plans.at(plan);
  long n = (long)p.n0 * p.n1 * p.n2;
  if (out != in) memcpy(out, in, sizeof(cufftDoubleComplex) * n);
  auto* d = reinterpret_cast<std::complex<double>*>(out);
  const int dims[3] = {p.n2, p.n1, p.n0};
  const long strides[3] = {1, p.n2, (long)p.n2 * p.n1};
  for (int a = 0; a < 3; ++a) {
    int m = dims[a];
    if (m == 1) continue;
    auto w = twiddles(m, direction);
    std::vector<std::complex<double>> tmp(m);
    for (long base = 0; base < n; ++base) {
      // base is the first element of a line along axis a
      if ((base / strides[a]) % m != 0) continue;
      dft_line(d + base, strides[a], m, direction, tmp, w);
    }
  }
  return CUFFT_SUCCESS;
}

cufftResult cufftDestroy(cufftHandle plan) {
  g_plans.erase(plan);
  return CUFFT_SUCCESS;
}

// --------------------------------------------------------------- cuRAND ---
namespace {
struct Gen {
  unsigned long long seed = 0;
  unsigned long long draws = 0;
};
std::map<int, Gen> g_gens;
int g_next_gen = 1;
}  // namespace

curandStatus_t curandCreateGenerator(curandGenerator_t* g, curandRngType) {
  *g = g_next_gen++;
  g_gens[*g] = Gen{};
  return 0;
}

curandStatus_t curandSetPseudoRandomGeneratorSeed(curandGenerator_t g, unsigned long long seed) {
  g_gens[g].seed = seed;
  return 0;
}

// One call per time step (src/runSchemeStokesLimit.cu:166): the noise of
// draw t = number of previous calls, from the oracle's Philox normals.
curandStatus_t curandGenerateNormalDouble(curandGenerator_t g, double* out, size_t n, double mean,
                                          double stddev) {
  Gen& G = g_gens[g];
  orc_noise(G.seed, G.draws, 0, (int64_t)n, out);
  for (size_t k = 0; k < n; ++k) out[k] = mean + stddev * out[k];
  G.draws++;
  return 0;
}

curandStatus_t curandDestroyGenerator(curandGenerator_t g) {
  g_gens.erase(g);
  return 0;
}
