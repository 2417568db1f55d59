/* fsl_oracle.h -- C interface of the FP64 CPU oracle for the Stokes-limit step.
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py as the checker.  The product never uses it.
 *
 * Parity status: pinned.  The restatement is checked against the reference's
 * own Stokes-limit kernels (src/stokesLimitFunctions.cu and friends) compiled
 * for the host by oracle/ref_cpu/build_ref.py into oracle/_ref/, on small
 * seeded cases (tests/test_oracle_vs_ref.py, tests/golden/).  The FFT and the
 * noise generator replace closed libraries (cuFFT, cuRAND) by published
 * algorithms; both sides of that comparison use them.
 *
 * Extensions over the reference (no reference counterpart, so not pinned by
 * it; pinned instead by known-answer tests): ORC_PAIR_SOFT, kernel == 4,
 * ORC_RFD_PAPER.
 *
 * Positions, forces and particle velocities are structure-of-arrays
 * x[0..np) | y[0..np) | z[0..np), as the reference's rx/ry/rz arrays.  Fields
 * are component-major [3][nc] with cell index x + y mx + z mx my.
 */
#ifndef FSL_ORACLE_H
#define FSL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_PAIR_NONE = 0, ORC_PAIR_TABLE_LJ = 1, ORC_PAIR_SOFT = 2 };
enum { ORC_RFD_REFERENCE = 0, ORC_RFD_PAPER = 1 };
/* ORC_SCHEME_MIDPOINT: stokesLimit (src/runSchemeStokesLimit.cu:163-285);
 * ORC_SCHEME_FIRST_ORDER: stokesLimitFirstOrder
 * (src/runSchemeStokesLimitFirstOrder.cu:163-241). */
/* ORC_SCHEME_QUASI2D / ORC_SCHEME_STOKES2D: the Gaussian-blob schemes of
 * keywords quasi2D and stokesLimit2D on an mx x my grid (mz = 1),
 * src/runSchemeQuasi2D.cu:20-260 with src/quasi2DFunctions.cu. */
/* ORC_SCHEME_INCOMPRESSIBLE: the fluctuating incompressible Navier-Stokes
 * solver of keyword incompressible (no particles),
 * src/runSchemeIncompressible.cu:20-155. */
enum { ORC_SCHEME_MIDPOINT = 0, ORC_SCHEME_FIRST_ORDER = 1, ORC_SCHEME_QUASI2D = 2,
       ORC_SCHEME_STOKES2D = 3, ORC_SCHEME_INCOMPRESSIBLE = 4 };

typedef struct orc_config {
  int32_t mx, my, mz;
  int32_t kernel;         /* 3 or 4 point Peskin kernel                  */
  double lx, ly, lz;
  double shearviscosity;
  double temperature;
  double dt;
  double cutoff;
  double extra_mobility;
  double soft_epsilon;
  uint64_t seed;
  int32_t pair;           /* ORC_PAIR_*                                  */
  int32_t rfd;            /* ORC_RFD_*                                   */
  int32_t nonbonded;      /* computeNonBondedForces                      */
  int32_t scheme;         /* ORC_SCHEME_*                                */
  /* quasi-2D family only */
  int32_t ndrift;         /* nDrift (noise count only)                   */
  int32_t use_rfd;        /* use_RFD                                     */
  int32_t predictor_corrector; /* predictorCorrector                     */
  int32_t pad_;
  double radius;          /* hydrodynamicRadius                          */
  double saffman_kc;      /* saffmanCutOffWaveNumber (stokesLimit2D)     */
  double saffman_width;   /* saffmanLayerWidth                           */
  double shear_amp;       /* viscosityMeasureAmplitude                   */
  double density;         /* densfluid (incompressible)                  */
} orc_config;

typedef struct orc_state orc_state;

orc_state* orc_create(const orc_config* cfg, int64_t np, const double* q);
void orc_destroy(orc_state* s);
int orc_set_bonds(orc_state* s, int64_t nbonds, const int32_t* bi, const int32_t* bj,
                  const double* bk, const double* br0, int64_t nfixed, const int32_t* fi,
                  const double* fk, const double* fr0, const double* fxyz);
/* Directed entries of the old bond-file format (bondedForcesVersion 1,
 * src/initializeBondedForcesOldVersion.cpp:41-238): entry b adds the spring
 * (bk, br0) towards particle bj[b] to particle bi[b] only (the file lists a
 * bond once from each end).  Tethers as orc_set_bonds. */
int orc_set_bonds_directed(orc_state* s, int64_t nentries, const int32_t* bi, const int32_t* bj,
                           const double* bk, const double* br0, int64_t nfixed, const int32_t* fi,
                           const double* fk, const double* fr0, const double* fxyz);
int orc_step(orc_state* s, int64_t nsteps);
void orc_get_positions(const orc_state* s, double* out);
void orc_set_positions(orc_state* s, const double* in);
void orc_get_predictor(const orc_state* s, double* out);
void orc_get_forces(const orc_state* s, double* out);
void orc_get_velocity(const orc_state* s, double* out);
/* Incompressible scheme: the initial staggered velocity [3][nc], projected
 * onto divergence-free fields as the scheme does before its first step
 * (src/runSchemeIncompressible.cu:82-96). */
void orc_set_velocity(orc_state* s, const double* v);
uint64_t orc_get_step(const orc_state* s);
void orc_set_step(orc_state* s, uint64_t t);
int orc_num_threads(void);

void orc_noise(uint64_t seed, uint64_t t, uint64_t first, int64_t count, double* out);
int orc_neighbor_grid(const orc_state* s, int32_t* dims3);
void orc_cell_list(orc_state* s, const double* q, int32_t* cell_of, int32_t* start,
                   int32_t* sorted);
void orc_forces(orc_state* s, const double* q, double* F);
void orc_spread(orc_state* s, const double* q, const double* F, double* f);
void orc_solve(orc_state* s, const double* W, double* v);
void orc_interp(orc_state* s, const double* q, const double* v, double* u);
void orc_build_W(orc_state* s, const double* f, int second, double* W);
void orc_fft3d(int mx, int my, int mz, int sign, double* re_im);
void orc_ljtable(orc_state* s, float* out);
float orc_tex_linear(const float* table, int n, float x);
double orc_delta3(double x);
double orc_delta4(double x);

#ifdef __cplusplus
}
#endif

#endif
