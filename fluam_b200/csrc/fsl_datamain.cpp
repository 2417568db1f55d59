// fsl_datamain.cpp -- the drop-in driver: fluam's data.main input contract and
// its particle output files, around the libfluamsl C ABI.
//
// Input  (src/loadDataMain.cu:173-683): whitespace-separated keywords, each
//   followed by a fixed number of values; '#' starts a comment to end of line;
//   an unknown keyword is an error ("ERROR INPUT FILE").  Every keyword of the
//   reference parser is accepted and consumes the same tokens; the ones that
//   the Stokes-limit path does not read are ignored.  Six keywords are new
//   (the reference parser would reject them): pairPotential lj|soft|none,
//   softEpsilon <eps>, kernelPoints 3|4, rfdMode reference|paper,
//   precision fixed64|float_atomic|fp64, observables 0|1 (3-D Stokes
//   schemes: <out>.observables, one line per sample: step*dt, msd, msd summed
//   over the steps, centre-of-mass displacement, total force, fluid momentum).
// Output (src/saveFunctionsSchemeStokesLimit.cu, src/saveParticles.cu:32-82,
//   src/saveSeed.cpp, src/saveTime.cpp, src/cudaDevice.cu):
//   <out>.data.main echo, <out>.cuda, <out>.seed, <out>.time,
//   <out>.particles and <out>.velocityParticles ("#NUMBER PARTICLES np", then
//   per sample a line step*dt and np lines "x y z", precision 15).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/fluamsl.h"

namespace {

struct Run {
  fsl_config cfg;
  int64_t numsteps = 0, relax = 0, samplefreq = 0, np = 0;
  bool have_seed = false;
  int loadparticles = 0;
  std::string coordinates, outputname, bondfile;
  bool bonded = false;
  int bond_version = 0;  // bondedForcesVersion: nonzero = the old file format
  // fluid output: saveFluid, saveVTK, savefreq, densfluid, pressureparameters
  int save_fluid = 0, save_vtk = 0;
  int64_t savefreq = 0;
  double densfluid = 0.0, pressure[3] = {0.0, 0.0, 0.0};
  // scheme flags that select another fluam scheme (src/main.cpp:36-105)
  bool stokesLimit = false, first_order = false, quasi2D = false, stokes2D = false, incomp = false;
  // initial fluid of the incompressible scheme (src/initializeFluid.cpp:28-82)
  int64_t initfluid = 0;
  bool setparticles = false;
  double v0[3] = {0.0, 0.0, 0.0};
  std::vector<std::string> other_schemes;
  std::string wordfile;
};

// Number of values that follow each keyword of the reference parser.
const std::map<std::string, int>& keyword_arity() {
  static const std::map<std::string, int> m = {
      {"particles", 1}, {"saffmanCutOffWaveNumber", 1}, {"saffmanLayerWidth", 1},
      {"viscosityMeasureAmplitude", 1}, {"identity_prefactor", 1}, {"gradTemperature", 1},
      {"soretCoefficient", 1}, {"backgroundvelocity", 3}, {"setDevice", 1},
      {"particlesdata", 1}, {"boundary", 1}, {"velocityboundary", 1},
      {"volumeboundaryconst", 1}, {"densfluid", 1}, {"shearviscosity", 1},
      {"bulkviscosity", 1}, {"temperature", 1}, {"thermostat", 0}, {"numsteps", 1},
      {"numstepsRelaxation", 1}, {"dt", 1}, {"samplefreq", 1}, {"savefreq", 1},
      {"pressureparameters", 3}, {"outputname", 1}, {"seed", 1}, {"cells", 3},
      {"celldimension", 3}, {"initfluid", 1}, {"checkVelocity", 1}, {"loadparticles", 1},
      {"coordinates", 1}, {"velocities", 1}, {"fluid", 1}, {"numberparticles", 1},
      {"mass", 1}, {"volumeParticle", 1}, {"cutoff", 1}, {"maxNumberPartInCell", 1},
      {"maxNumberPartInCellNonBonded", 1}, {"dDensity", 1}, {"omega", 1},
      {"waveSourceIndex", 1}, {"saveFluid", 1}, {"saveVTK", 1}, {"ghost", 0},
      {"bondedForces", 1}, {"bondedForcesVersion", 1}, {"computeNonBondedForces", 1},
      {"binaryMixture", 0}, {"diffusion", 1}, {"massSpecies0", 1}, {"massSpecies1", 1},
      {"concentration", 1}, {"binaryMixtureWall", 0}, {"concentrationWall", 2},
      {"vxWall", 2}, {"vyWall", 2}, {"vzWall", 2}, {"densityWall", 2},
      {"giantFluctuations", 0}, {"continuousGradient", 0}, {"incompressible", 0},
      {"incompressibleBoundaryRK2", 0}, {"quasiNeutrallyBuoyant", 0},
      {"quasiNeutrallyBuoyant2D", 0}, {"quasiNeutrallyBuoyant4pt2D", 0}, {"quasi2D", 0},
      {"hydrodynamicRadius", 1}, {"nDrift", 1}, {"stokesLimit2D", 0},
      {"predictorCorrector", 1}, {"sampleHydroGrid", 1}, {"cellsHydroGrid", 2},
      {"greenParticles", 2}, {"use_RFD", 1}, {"IMEXRK", 0},
      {"incompressibleBinaryMixture", 0}, {"incompressibleBinaryMixtureMidPoint", 0},
      {"particlesWall", 0}, {"freeEnergyCompressibleParticles", 0}, {"omega0", 1},
      {"semiImplicitCompressibleParticles", 0}, {"momentumCoupling", 0},
      {"stokesLimitFirstOrder", 0}, {"stokesLimit", 0}, {"extraMobility", 1},
      // extensions of this build
      {"pairPotential", 1}, {"softEpsilon", 1}, {"kernelPoints", 1}, {"rfdMode", 1},
      {"precision", 1}, {"observables", 1}, {"savedensity", -1}};
  return m;
}

int parse(const char* path, Run& r, std::string& err) {
  fsl_config_defaults(&r.cfg);
  std::ifstream in(path);
  if (!in) {
    err = std::string("cannot open ") + path;
    return FSL_E_IO;
  }
  // wordfile echo exactly as src/loadDataMain.cu:313-317
  {
    std::string line;
    while (!in.eof()) {
      std::getline(in, line);
      r.wordfile += line + "\n";
    }
  }
  in.close();
  in.open(path);
  const auto& ar = keyword_arity();
  std::string word, oldword;
  int64_t thermostat = 0;
  in >> word;
  while (!in.eof()) {
    if (!word.empty() && word[0] == '#') {
      std::getline(in, word);
    } else {
      auto it = ar.find(word);
      if (it == ar.end()) {
        err = "ERROR INPUT FILE; LAST WORD READED: " + oldword + " (unknown keyword '" + word + "')";
        return FSL_E_INPUT;
      }
      std::vector<std::string> vals;
      int n = it->second;
      if (word == "savedensity") {
        std::string v;
        in >> v;
        if (v == "1") {
          int64_t ns = 0;
          in >> ns;
          for (int64_t k = 0; k < ns; ++k) in >> v;
        } else {
          std::getline(in, v);
        }
        n = 0;
      }
      for (int k = 0; k < n; ++k) {
        std::string v;
        in >> v;
        vals.push_back(v);
      }
      auto D = [&](int k) { return std::strtod(vals[k].c_str(), nullptr); };
      auto I = [&](int k) { return (int64_t)std::strtoll(vals[k].c_str(), nullptr, 10); };
      fsl_config& c = r.cfg;
      if (word == "cells") {
        c.mx = (int)I(0);
        c.my = (int)I(1);
        c.mz = (int)I(2);
      } else if (word == "celldimension") {
        c.lx = D(0);
        c.ly = D(1);
        c.lz = D(2);
      } else if (word == "shearviscosity") {
        c.shearviscosity = D(0);
      } else if (word == "temperature") {
        c.temperature = D(0);
      } else if (word == "dt") {
        c.dt = D(0);
      } else if (word == "cutoff") {
        c.cutoff = D(0);
      } else if (word == "numsteps") {
        r.numsteps = I(0);
      } else if (word == "numstepsRelaxation") {
        r.relax = I(0);
      } else if (word == "samplefreq") {
        r.samplefreq = I(0);
      } else if (word == "seed") {
        c.seed = (uint64_t)I(0);
        r.have_seed = true;
      } else if (word == "outputname") {
        r.outputname = vals[0];
      } else if (word == "numberparticles") {
        r.np = I(0);
      } else if (word == "loadparticles") {
        r.loadparticles = (int)I(0);
      } else if (word == "coordinates") {
        r.coordinates = vals[0];
      } else if (word == "bondedForces") {
        r.bonded = true;
        r.bondfile = vals[0];
      } else if (word == "bondedForcesVersion") {
        r.bond_version = (int)I(0);
      } else if (word == "computeNonBondedForces") {
        c.nonbonded = (int)I(0);
      } else if (word == "extraMobility") {
        c.extra_mobility = D(0);
      } else if (word == "saveFluid") {
        r.save_fluid = (int)I(0);
      } else if (word == "saveVTK") {
        r.save_vtk = (int)I(0);
      } else if (word == "savefreq") {
        r.savefreq = I(0);
      } else if (word == "densfluid") {
        r.densfluid = D(0);
      } else if (word == "pressureparameters") {
        r.pressure[0] = D(0);
        r.pressure[1] = D(1);
        r.pressure[2] = D(2);
      } else if (word == "setDevice") {
        c.device = (int)I(0);
      } else if (word == "stokesLimit") {
        r.stokesLimit = true;
      } else if (word == "stokesLimitFirstOrder") {
        r.first_order = true;
      } else if (word == "thermostat") {
        thermostat = 1;
      } else if (word == "pairPotential") {
        if (vals[0] == "lj") c.pair = FSL_PAIR_TABLE_LJ;
        else if (vals[0] == "soft") c.pair = FSL_PAIR_SOFT;
        else if (vals[0] == "none") c.pair = FSL_PAIR_NONE;
        else {
          err = "pairPotential must be lj, soft or none";
          return FSL_E_INPUT;
        }
      } else if (word == "softEpsilon") {
        c.soft_epsilon = D(0);
      } else if (word == "kernelPoints") {
        c.kernel = (int)I(0);
      } else if (word == "rfdMode") {
        if (vals[0] == "reference") c.rfd = FSL_RFD_REFERENCE;
        else if (vals[0] == "paper") c.rfd = FSL_RFD_PAPER;
        else {
          err = "rfdMode must be reference or paper";
          return FSL_E_INPUT;
        }
      } else if (word == "observables") {
        c.observables = std::atoi(vals[0].c_str());
      } else if (word == "precision") {
        if (vals[0] == "fixed64") c.precision = FSL_PRECISION_FIXED64;
        else if (vals[0] == "float_atomic") c.precision = FSL_PRECISION_FLOAT_ATOMIC;
        else if (vals[0] == "fp64") c.precision = FSL_PRECISION_FP64;
        else {
          err = "precision must be fixed64, float_atomic or fp64";
          return FSL_E_INPUT;
        }
      } else if (word == "continuousGradient" || word == "giantFluctuations" ||
                 word == "binaryMixtureWall" || word == "binaryMixture" ||
                 word == "particlesWall" || word == "freeEnergyCompressibleParticles" ||
                 word == "semiImplicitCompressibleParticles" || word == "momentumCoupling" ||
                 word == "incompressibleBinaryMixture" ||
                 word == "incompressibleBinaryMixtureMidPoint" ||
                 word == "quasiNeutrallyBuoyant" || word == "quasiNeutrallyBuoyant2D" ||
                 word == "quasiNeutrallyBuoyant4pt2D") {
        r.other_schemes.push_back(word);
      } else if (word == "incompressible") {
        r.incomp = true;
      } else if (word == "particles") {
        r.setparticles = I(0) != 0;
      } else if (word == "initfluid") {
        r.initfluid = I(0);
      } else if (word == "backgroundvelocity") {
        r.v0[0] = D(0);
        r.v0[1] = D(1);
        r.v0[2] = D(2);
      } else if (word == "quasi2D") {
        r.quasi2D = true;
      } else if (word == "stokesLimit2D") {
        r.stokes2D = true;
      } else if (word == "hydrodynamicRadius") {
        c.radius = D(0);
      } else if (word == "nDrift") {
        c.ndrift = (int)I(0);
      } else if (word == "use_RFD") {
        c.use_rfd = (int)I(0);
      } else if (word == "predictorCorrector") {
        c.predictor_corrector = (int)I(0);
      } else if (word == "saffmanCutOffWaveNumber") {
        c.saffman_kc = D(0);
      } else if (word == "saffmanLayerWidth") {
        c.saffman_width = D(0);
      } else if (word == "viscosityMeasureAmplitude") {
        c.shear_amp = D(0);
      }
    }
    oldword = word;
    in >> word;
  }
  // the reference's scheme precedence (src/main.cpp:36-99): all of these come
  // before stokesLimit in its if-chain
  if (thermostat) r.other_schemes.push_back("thermostat");
  // stokesLimitFirstOrder precedes stokesLimit (src/main.cpp:94-99).  With
  // stokesLimitFirstOrder alone the reference never uploads the cell-centre
  // coordinates (src/initializeFluidIncompressibleGPU.cu:27 tests stokesLimit
  // only) and its kernels read uninitialised device memory; this build uses
  // the cell centres in both cases, which is what the reference computes when
  // the file holds both keywords.
  if (r.first_order) r.cfg.scheme = FSL_SCHEME_FIRST_ORDER;
  // quasi2D / stokesLimit2D precede both (src/main.cpp:91-93); with both
  // keywords the quasi2D branches win (src/createCellsQuasi2DGPU.cu:53-61,
  // src/runSchemeQuasi2D.cu:186-205)
  if (r.quasi2D) r.cfg.scheme = FSL_SCHEME_QUASI2D;
  else if (r.stokes2D) r.cfg.scheme = FSL_SCHEME_STOKES2D;
  // incompressible comes before all of them in the reference's chain, and
  // with particles it selects another scheme (src/main.cpp:70-75); densfluid
  // is its fluid density
  if (r.incomp && r.setparticles) r.other_schemes.push_back("incompressibleBoundary");
  if (r.incomp) {
    r.cfg.scheme = FSL_SCHEME_INCOMPRESSIBLE;
    r.cfg.density = r.densfluid;
  }
  return FSL_OK;
}

bool read_coordinates(const std::string& file, std::vector<double>& q, int64_t& np) {
  // src/createParticles.cpp:81-101: np then np lines "x y z"
  std::ifstream f(file);
  if (!f) return false;
  f >> np;
  if (!f || np < 0) return false;
  std::vector<double> x(np), y(np), z(np);
  for (int64_t i = 0; i < np; ++i) f >> x[i] >> y[i] >> z[i];
  if (!f) return false;
  q.resize(3 * np);
  for (int64_t i = 0; i < np; ++i) {
    q[i] = x[i];
    q[np + i] = y[i];
    q[2 * np + i] = z[i];
  }
  return true;
}

void simple_cubic(const fsl_config& c, int64_t np, std::vector<double>& q, int dimension) {
  // src/simpleCubic.cpp:25-63: a lattice in 3-D, or a single layer in 2-D
  // (which the filling loop may still stack)
  double lx = c.lx, ly = c.ly, lz = c.lz;
  double sigma;
  int nz;
  if (dimension == 3) {
    sigma = std::pow(lx * ly * lz / (np), 1. / 3.);
    nz = (int(lz / sigma) ? int(lz / sigma) : 1);
  } else {
    sigma = std::sqrt(lx * ly / np);
    nz = 1;
  }
  int nx = (int(lx / sigma) ? int(lx / sigma) : 1);
  int ny = (int(ly / sigma) ? int(ly / sigma) : 1);
  while ((int64_t)nx * ny * nz < np) {
    if ((int64_t)nx * ny * nz < np) nx++;
    if ((int64_t)nx * ny * nz < np) ny++;
    if ((int64_t)nx * ny * nz < np) nz++;
  }
  double dx = lx / double(nx), dy = ly / double(ny), dz = lz / double(nz);
  q.assign(3 * np, 0.0);
  int64_t n = 0;
  for (int i = 0; i <= nz - 1; i++)
    for (int j = 0; j <= ny - 1; j++)
      for (int k = 0; k <= nx - 1; k++)
        if (n < np) {
          n = n + 1;
          q[n - 1] = (k + 0.5) * dx - lx / 2.;
          q[np + n - 1] = (j + 0.5) * dy - ly / 2.;
          q[2 * np + n - 1] = (i + 0.5) * dz - lz / 2.;
        }
}

struct Bonds {
  std::vector<int32_t> bi, bj, fi;
  std::vector<double> k, r0, fk, fr0, fxyz;
};

bool read_bonds(const std::string& file, Bonds& b) {
  // src/initializeBondedForces.cpp:31-150 (format in bin/inputfiles/README:60-108)
  std::ifstream f(file);
  if (!f) return false;
  int64_t n = 0;
  f >> n;
  if (!f || n < 0) return false;
  for (int64_t k = 0; k < n; ++k) {
    int i1, i2;
    double ks, r0;
    f >> i1 >> i2 >> ks >> r0;
    b.bi.push_back(i1);
    b.bj.push_back(i2);
    b.k.push_back(ks);
    b.r0.push_back(r0);
  }
  int64_t nf = 0;
  f >> nf;
  if (!f || nf < 0) return false;
  for (int64_t k = 0; k < nf; ++k) {
    int i1;
    double ks, r0, x, y, z;
    f >> i1 >> ks >> r0 >> x >> y >> z;
    b.fi.push_back(i1);
    b.fk.push_back(ks);
    b.fr0.push_back(r0);
    b.fxyz.push_back(x);
    b.fxyz.push_back(y);
    b.fxyz.push_back(z);
  }
  return (bool)f;
}

// The old bond-file format (bondedForcesVersion != 0,
// src/initializeBondedForcesOldVersion.cpp:41-238): the particle-particle
// count counts every bond twice, each line "i j k r0" acts on i only and the
// lines are sorted by i; then the tethers "i k r0 x y z".  Deliberate
// differences: an unsorted particle-particle list is an input error here
// (the reference prints "bad sorting" and goes on with tables it never
// filled), and a particle's tethers are grouped in file order (the
// reference's first pass never updates its running index, so it misplaces
// a particle's second and later tethers).
bool read_bonds_old(const std::string& file, Bonds& b, std::string& why) {
  std::ifstream f(file);
  if (!f) {
    why = "cannot open";
    return false;
  }
  int64_t n = 0;
  f >> n;
  if (!f || n < 0) {
    why = "bad particle-particle count";
    return false;
  }
  int prev = -1;
  for (int64_t k = 0; k < n; ++k) {
    int i1, i2;
    double ks, r0;
    f >> i1 >> i2 >> ks >> r0;
    if (!f) {
      why = "short particle-particle list";
      return false;
    }
    if (i1 < prev) {
      why = "bad sorting in bonded Forces Particle-Particle";
      return false;
    }
    prev = i1;
    b.bi.push_back(i1);
    b.bj.push_back(i2);
    b.k.push_back(ks);
    b.r0.push_back(r0);
  }
  int64_t nf = 0;
  f >> nf;
  if (!f || nf < 0) {
    why = "bad particle-fixed point count";
    return false;
  }
  for (int64_t k = 0; k < nf; ++k) {
    int i1;
    double ks, r0, x, y, z;
    f >> i1 >> ks >> r0 >> x >> y >> z;
    b.fi.push_back(i1);
    b.fk.push_back(ks);
    b.fr0.push_back(r0);
    b.fxyz.push_back(x);
    b.fxyz.push_back(y);
    b.fxyz.push_back(z);
  }
  if (!f) why = "short particle-fixed point list";
  return (bool)f;
}

void write_cuda_file(const std::string& out, int setDevice) {
  // src/cudaDevice.cu:23-83
  std::ofstream f(out + ".cuda");
  int count = 0, drv = 0, rt = 0;
  cudaGetDeviceCount(&count);
  f << std::endl << "cudaGetDeviceCount     " << count << std::endl;
  for (int i = 0; i < count; i++) {
    cudaDeviceProp p;
    cudaGetDeviceProperties(&p, i);
    f << std::endl << "Device " << i << ": version " << p.major << " " << p.minor << std::endl;
    f << p.name << std::endl;
    cudaDriverGetVersion(&drv);
    f << "Driver version                  " << drv << std::endl;
    cudaRuntimeGetVersion(&rt);
    f << "Runtime version                 " << rt << std::endl;
    f << "Multiprocessors                 " << p.multiProcessorCount << std::endl;
    f << "Global memory (bytes)           " << p.totalGlobalMem << std::endl;
    f << "Constant memory (bytes)         " << p.totalConstMem << std::endl;
    f << "Shared memory per block (bytes) " << p.sharedMemPerBlock << std::endl;
    f << "Registers per block             " << p.regsPerBlock << std::endl;
    f << "Warp size                       " << p.warpSize << std::endl;
    f << "Maximum threads per block       " << p.maxThreadsPerBlock << std::endl;
    int clk = 0;
    cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, i);
    f << "Clock rate (GHz)                " << clk * 1e-6 << std::endl;
    int mode = 0;
    cudaDeviceGetAttribute(&mode, cudaDevAttrComputeMode, i);
    f << "Compute Mode                    " << mode << std::endl;
  }
  if (setDevice >= 0) {
    cudaSetDevice(setDevice);
    int d = 0;
    cudaGetDevice(&d);
    f << std::endl << std::endl << std::endl;
    f << "Device selected " << d << std::endl;
  }
  f << std::endl;
}

void write_sample(std::ofstream& f, int64_t np, const std::vector<double>& a, double t) {
  f << t << std::endl;
  for (int64_t i = 0; i < np; ++i) f << a[i] << " " << a[np + i] << " " << a[2 * np + i] << std::endl;
}

// ASCII number stream of the legacy VTK layout: "%20.12e " per value, a line
// break after every ninth value of a run, a break before a new section when
// the current line is open.
struct VtkText {
  FILE* f;
  int col = 0;
  void end_line() {
    std::fputc('\n', f);
    col = 0;
  }
  void section() {
    if (col != 0) end_line();
  }
  void num(double x) {
    std::fprintf(f, "%20.12e ", x);
    if ((col++ % 9) == 8) end_line();
  }
};

// One snapshot name: <out>.<index>.fluid.vtk (src/saveFluidVTK.cu:40-47)
std::string vtk_name(const std::string& out, int64_t index) {
  return out + "." + std::to_string(index) + ".fluid.vtk";
}

int fluid_outputs(fsl_handle* h, const Run& r, int final_call, int64_t step) {
  const int mx = r.cfg.mx, my = r.cfg.my, mz = r.cfg.mz;
  std::vector<double> v(3 * (size_t)mx * my * mz);
  int rc = fsl_get_velocity_f64(h, v.data());
  if (rc) return rc;
  if (!final_call) {
    return fsl_write_fluid_vtk(vtk_name(r.outputname, step / r.savefreq).c_str(), mx, my, mz, v.data());
  }
  if (r.save_fluid) {
    rc = fsl_write_fluid_final((r.outputname + ".fluidFinalConfiguration").c_str(), &r.cfg,
                               r.densfluid, r.pressure, 0, v.data());
    if (rc) return rc;
  }
  if (r.save_vtk) rc = fsl_write_fluid_vtk((r.outputname + ".fluid.vtk").c_str(), mx, my, mz, v.data());
  return rc;
}

// Running averages of the fluid temperature diagnostic
// (src/temperature.cu:32-205, indices 1 and 2).
struct FluidTemperature {
  double sigma = 0, mean = 0, txm = 0, tym = 0, tzm = 0;
  // per sample: kinetic temperature of the staggered velocity about its mean
  void sample(const Run& r, const std::vector<double>& v, int64_t step) {
    const int64_t nc = (int64_t)r.cfg.mx * r.cfg.my * r.cfg.mz;
    const double vol = (r.cfg.lx / r.cfg.mx) * (r.cfg.ly / r.cfg.my) * (r.cfg.lz / r.cfg.mz);
    const double rho = r.cfg.density;
    const int64_t n = step / r.samplefreq;
    double m[3] = {0, 0, 0}, mass = 0;
    for (int64_t i = 0; i < nc; ++i) {
      for (int a = 0; a < 3; ++a) m[a] += v[a * nc + i];
      mass += vol * rho;
    }
    for (int a = 0; a < 3; ++a) m[a] /= double(nc);
    double t[3] = {0, 0, 0}, p[3] = {0, 0, 0};
    for (int64_t i = 0; i < nc; ++i)
      for (int a = 0; a < 3; ++a) {
        const double d = v[a * nc + i] - m[a];
        t[a] += 0.5 * vol * (rho + rho) * d * d;
        p[a] += 0.5 * vol * (rho + rho) * v[a * nc + i];
      }
    for (int a = 0; a < 3; ++a) t[a] /= double(nc);
    const double tt = (t[0] + t[1] + t[2]) / 3.;
    const double T = r.cfg.temperature;
    sigma += (tt - T) * (tt - T);
    mean += tt;
    txm += t[0];
    tym += t[1];
    tzm += t[2];
    std::cout << "MASS FLUID    " << mass << std::endl;
    std::cout << "TEMPERATURE FLUID " << tt << " " << mean / double(n) << " "
              << (mean / double(n) - T) / T << " " << std::sqrt(sigma / double(n)) / T << "  " << n
              << std::endl;
    std::cout << "tx                " << t[0] << " " << txm / double(n) << std::endl;
    std::cout << "ty                " << t[1] << " " << tym / double(n) << std::endl;
    std::cout << "tz                " << t[2] << " " << tzm / double(n) << std::endl;
    std::cout.precision(15);
    std::cout << "PX " << p[0] << std::endl << "PY " << p[1] << std::endl << "PZ " << p[2] << std::endl
              << std::endl;
    std::cout.precision(6);
  }
  // <out>.temperature at the end, momenta of the last sampled field
  void close(const Run& r, const std::vector<double>& v, int64_t step) const {
    const int64_t nc = (int64_t)r.cfg.mx * r.cfg.my * r.cfg.mz;
    const double vol = (r.cfg.lx / r.cfg.mx) * (r.cfg.ly / r.cfg.my) * (r.cfg.lz / r.cfg.mz);
    const double rho = r.cfg.density, T = r.cfg.temperature;
    const int64_t n = step / r.samplefreq;
    std::ofstream f(r.outputname + ".temperature");
    f.precision(15);
    f << "TEMPERATURE FLUID " << mean / double(n) << " " << (mean / double(n) - T) / T << " "
      << std::sqrt(sigma / double(n)) / T << "  " << n << std::endl;
    f << "tx                " << txm / double(n) << std::endl;
    f << "ty                " << tym / double(n) << std::endl;
    f << "tz                " << tzm / double(n) << std::endl;
    double p[3] = {0, 0, 0}, mass = 0;
    for (int64_t i = 0; i < nc; ++i) {
      for (int a = 0; a < 3; ++a) p[a] += 0.5 * vol * (rho + rho) * v[a * nc + i];
      mass += vol * rho;
    }
    f << "PX " << p[0] << std::endl;
    f << "PY " << p[1] << std::endl;
    f << "PZ " << p[2] << std::endl << std::endl;
    f << "MASS FLUID    " << mass << std::endl << std::endl;
  }
};

// schemeIncompressible + runSchemeIncompressible (src/schemeIncompressible.cu:
// 23-55, src/runSchemeIncompressible.cu:20-155): the initial field (a uniform
// background velocity, initfluid 0; the other initfluid choices draw from the
// reference's host generator and are not supported), samples after every
// samplefreq-th step, the temperature diagnostic and the final fluid file.
int run_incompressible(Run& r) {
  if (r.initfluid != 0) {
    std::cout << "ERROR: the incompressible scheme supports initfluid 0 (background velocity) only"
              << std::endl;
    return FSL_E_INPUT;
  }
  const int64_t nc = (int64_t)r.cfg.mx * r.cfg.my * r.cfg.mz;
  std::vector<double> v(3 * nc);
  for (int a = 0; a < 3; ++a) std::fill(v.begin() + a * nc, v.begin() + (a + 1) * nc, r.v0[a]);
  fsl_handle* h = nullptr;
  int rc = fsl_create(&r.cfg, 0, nullptr, &h);
  if (!rc) rc = fsl_set_velocity_f64(h, v.data());
  if (rc) {
    std::cout << "ERROR: " << fsl_last_error() << std::endl;
    if (h) fsl_destroy(h);
    return rc;
  }
  {
    std::ofstream fs(r.outputname + ".seed");
    fs << r.cfg.seed << std::endl;
  }
  time_t t0 = time(NULL);
  FluidTemperature temp;
  // the host copy the final files read: the initial field until a sample
  std::vector<double> last = v;
  int64_t step = -r.relax;
  while (step < r.numsteps) {
    int64_t next = r.numsteps;
    const int64_t s0 = step + 1;
    int64_t cand = s0 <= 0 ? r.samplefreq : ((s0 + r.samplefreq - 1) / r.samplefreq) * r.samplefreq;
    if (cand < next) next = cand;
    rc = fsl_step(h, next - step);
    if (rc) break;
    step = next;
    if (!(step % r.samplefreq) && step > 0) {
      std::cout << "INCOMPRESSIBLE " << step << std::endl;
      if ((rc = fsl_sync(h)) || (rc = fsl_get_velocity_f64(h, last.data()))) break;
      temp.sample(r, last, step);
    }
  }
  if (!rc) rc = fsl_sync(h);
  time_t t1 = time(NULL) - t0;
  std::cout << std::endl << "TIME RUN_GPU                       " << t1 << std::endl << std::endl;
  {
    std::ofstream ft(r.outputname + ".time");
    ft << "TIME RUN GPU     " << t1 << std::endl;
  }
  if (!rc) {
    temp.close(r, last, step);
    const double p3[3] = {r.pressure[0], r.pressure[1], r.pressure[2]};
    rc = fsl_write_fluid_final((r.outputname + ".fluidFinalConfiguration").c_str(), &r.cfg,
                               r.densfluid, p3, 0, last.data());
  }
  if (rc) std::cout << "ERROR: " << fsl_last_error() << std::endl;
  fsl_destroy(h);
  if (!rc) std::cout << "END" << std::endl;
  return rc;
}

}  // namespace

extern "C" int fsl_parse_data_main(const char* path, fsl_config* cfg, int64_t* numsteps,
                                   int64_t* samplefreq, int64_t* relax, int64_t* np) {
  if (!path || !cfg) return FSL_E_ARG;
  Run r;
  std::string err;
  int rc = parse(path, r, err);
  if (rc) {
    std::cerr << err << std::endl;
    return rc;
  }
  *cfg = r.cfg;
  if (numsteps) *numsteps = r.numsteps;
  if (samplefreq) *samplefreq = r.samplefreq;
  if (relax) *relax = r.relax;
  if (np) *np = r.np;
  return FSL_OK;
}

extern "C" int fsl_run_data_main(const char* path) {
  Run r;
  std::string err;
  int rc = parse(path ? path : "data.main", r, err);
  if (rc) {
    std::cout << err << std::endl;
    return rc;
  }
  // echo of the input (src/loadDataMain.cu:672-676)
  {
    std::ofstream fo(r.outputname + ".data.main");
    fo << r.wordfile << std::endl;
  }
  std::cout << "READ " << (path ? path : "data.main") << " :                DONE" << std::endl;
  if (!r.other_schemes.empty() ||
      !(r.stokesLimit || r.first_order || r.quasi2D || r.stokes2D || r.incomp)) {
    std::cout << "ERROR: this build runs the stokesLimit, stokesLimitFirstOrder, quasi2D, "
                 "stokesLimit2D and incompressible schemes only"
              << (r.other_schemes.empty() ? std::string(" (keyword stokesLimit missing)")
                                          : " (found " + r.other_schemes[0] + ")")
              << std::endl;
    return FSL_E_INPUT;
  }
  if (r.samplefreq <= 0) {
    // the reference divides by samplefreq (src/runSchemeStokesLimit.cu:280)
    std::cout << "ERROR: samplefreq must be > 0" << std::endl;
    return FSL_E_INPUT;
  }
  write_cuda_file(r.outputname, r.cfg.device);
  // src/initializeRandomNumber.cpp:23-36
  if (!r.have_seed) {
    uint64_t s = (uint64_t)time(0);
    r.cfg.seed = s % 18671;
  }
  if (r.incomp) return run_incompressible(r);
  // particles (src/createParticles.cpp:39-102)
  std::vector<double> q;
  int64_t np = r.np;
  if (r.loadparticles == 1) {
    if (r.coordinates.empty()) {
      std::cout << "ERROR NO PARTICLESCOOR FILE FOUND" << std::endl;
      return FSL_E_INPUT;
    }
    if (!read_coordinates(r.coordinates, q, np)) {
      std::cout << "ERROR reading coordinates file " << r.coordinates << std::endl;
      return FSL_E_IO;
    }
  } else {
    if (np <= 0) {
      std::cout << "ERROR: numberparticles must be > 0" << std::endl;
      return FSL_E_INPUT;
    }
    // src/createParticles.cpp:53-58
    simple_cubic(r.cfg, np, q,
                 r.cfg.scheme == FSL_SCHEME_QUASI2D || r.cfg.scheme == FSL_SCHEME_STOKES2D ? 2 : 3);
  }
  fsl_handle* h = nullptr;
  rc = fsl_create(&r.cfg, np, q.data(), &h);
  if (rc) {
    std::cout << "ERROR: " << fsl_last_error() << std::endl;
    return rc;
  }
  if (r.bonded) {
    Bonds b;
    std::string why;
    if (r.bond_version ? !read_bonds_old(r.bondfile, b, why) : !read_bonds(r.bondfile, b)) {
      std::cout << "ERROR reading bondedForces file " << r.bondfile << (why.empty() ? "" : ": ")
                << why << std::endl;
      fsl_destroy(h);
      return FSL_E_IO;
    }
    rc = (r.bond_version ? fsl_load_bonds_directed : fsl_load_bonds)(
        h, (int64_t)b.bi.size(), b.bi.data(), b.bj.data(), b.k.data(), b.r0.data(),
        (int64_t)b.fi.size(), b.fi.data(), b.fk.data(), b.fr0.data(), b.fxyz.data());
    if (rc) {
      std::cout << "ERROR: " << fsl_last_error() << std::endl;
      fsl_destroy(h);
      return rc;
    }
  }
  {
    std::ofstream fs(r.outputname + ".seed");
    fs << r.cfg.seed << std::endl;
  }
  time_t t0 = time(NULL);
  // the first-order scheme writes no .velocityParticles (src/saveParticles.cu:43-46)
  // .velocityParticles: the midpoint scheme writes F^{n+1/2}; the first-order
  // scheme and quasi2D write none; stokesLimit2D writes the particle velocity
  // array, which that scheme never sets, so zeros (src/saveParticles.cu:43-47,
  // src/gpuToHostStokesLimit.cu:41-43)
  const bool q2 = r.cfg.scheme == FSL_SCHEME_QUASI2D || r.cfg.scheme == FSL_SCHEME_STOKES2D;
  const bool write_forces = r.cfg.scheme == FSL_SCHEME_MIDPOINT || r.cfg.scheme == FSL_SCHEME_STOKES2D;
  std::ofstream fp(r.outputname + ".particles"), fv;
  if (write_forces) fv.open(r.outputname + ".velocityParticles");
  fp.precision(15);
  fv.precision(15);
  std::ofstream fo;
  if (r.cfg.observables && !q2) {
    fo.open(r.outputname + ".observables");
    fo.precision(15);
    fo << "# time msd msd_sum dx dy dz Fx Fy Fz Px Py Pz" << std::endl;
  }
  fp << "#NUMBER PARTICLES " << np << std::endl;
  if (write_forces) fv << "#NUMBER PARTICLES " << np << std::endl;
  std::vector<double> pos(3 * np), frc(3 * np);
  int64_t step = -r.relax;
  if (q2) {
    // src/runSchemeQuasi2D.cu:99-252: a sample at the top of every step with
    // step >= 0 and step % samplefreq == 0, and one after the last step
    auto sample = [&]() -> int {
      std::cout << (r.cfg.scheme == FSL_SCHEME_QUASI2D ? "Quasi 2D " : "stokesLimit 2D ") << step
                << std::endl;
      int e = fsl_sync(h);
      if (e) {
        std::cout << "ERROR IN KERNEL: " << fsl_last_error() << std::endl;
        return e;
      }
      if ((e = fsl_get_positions(h, pos.data()))) return e;
      write_sample(fp, np, pos, step * r.cfg.dt);
      if (write_forces) write_sample(fv, np, std::vector<double>(3 * np, 0.0), step * r.cfg.dt);
      return FSL_OK;
    };
    while (step < r.numsteps && !rc) {
      if (step >= 0 && step % r.samplefreq == 0 && (rc = sample())) break;
      int64_t next = step < 0 ? 0 : (step / r.samplefreq + 1) * r.samplefreq;
      if (next > r.numsteps) next = r.numsteps;
      rc = fsl_step(h, next - step);
      if (rc) break;
      step = next;
    }
    if (!rc && step % r.samplefreq == 0) rc = sample();
  }
  // src/runSchemeStokesLimit.cu:83, 163-285
  while (!q2 && step < r.numsteps) {
    // next step index s > step with s % samplefreq == 0 and s > 0, or the end
    int64_t next = r.numsteps;
    int64_t s0 = step + 1;
    int64_t cand = ((s0 + r.samplefreq - 1) / r.samplefreq) * r.samplefreq;
    if (s0 <= 0) cand = r.samplefreq;
    if (cand < next) next = cand;
    rc = fsl_step(h, next - step);
    if (rc) break;
    step = next;
    if (!(step % r.samplefreq) && step > 0) {
      std::cout << "Stokes Limit  " << step << std::endl;
      rc = fsl_sync(h);
      if (rc) {
        std::cout << "ERROR IN KERNEL: " << fsl_last_error() << std::endl;
        break;
      }
      if ((rc = fsl_get_positions(h, pos.data())) || (rc = fsl_get_forces(h, frc.data()))) break;
      write_sample(fp, np, pos, step * r.cfg.dt);
      if (write_forces) write_sample(fv, np, frc, step * r.cfg.dt);
      if (r.cfg.observables) {
        fsl_observables o;
        if ((rc = fsl_get_observables(h, &o))) break;
        fo << step * r.cfg.dt << " " << o.msd << " " << o.msd_sum;
        for (double x : o.displacement) fo << " " << x;
        for (double x : o.force) fo << " " << x;
        for (double x : o.momentum) fo << " " << x;
        fo << std::endl;
      }
      // fluid snapshots at sample steps that are multiples of savefreq, as
      // the reference's other schemes do (src/saveFunctionsSchemeIncompressibleBoundary.cu:43-46)
      if (r.save_vtk && r.savefreq > 0 && step % r.savefreq == 0 &&
          (rc = fluid_outputs(h, r, 0, step)))
        break;
    }
  }
  if (rc) std::cout << "ERROR: " << fsl_last_error() << std::endl;
  if (!rc) rc = fsl_sync(h);
  // final fluid files (src/saveFunctionsSchemeIncompressibleBoundary.cu:57-59)
  if (!rc && (r.save_fluid || r.save_vtk)) {
    rc = fluid_outputs(h, r, 1, step);
    if (rc) std::cout << "ERROR: " << fsl_last_error() << std::endl;
  }
  time_t t1 = time(NULL) - t0;
  std::cout << std::endl << "TIME RUN_GPU                       " << t1 << std::endl << std::endl;
  {
    std::ofstream ft(r.outputname + ".time");
    ft << "TIME RUN GPU     " << t1 << std::endl;
  }
  fsl_destroy(h);
  if (!rc) std::cout << "END" << std::endl;
  return rc;
}

extern "C" int fsl_write_fluid_final(const char* path, const fsl_config* cfg, double density,
                                     const double* pressure3, int32_t thermostat, const double* v) {
  if (!path || !cfg || !v) return FSL_E_ARG;
  std::ofstream f(path);
  if (!f) return FSL_E_IO;
  const int64_t nc = (int64_t)cfg->mx * cfg->my * cfg->mz;
  const double p0 = pressure3 ? pressure3[0] : 0.0, p1 = pressure3 ? pressure3[1] : 0.0,
               p2 = pressure3 ? pressure3[2] : 0.0;
  f.precision(15);
  f << "Number of cells " << nc << std::endl;
  f << "mx my mz" << std::endl;
  f << cfg->mx << " " << cfg->my << " " << cfg->mz << std::endl;
  f << "lx ly lz" << std::endl;
  f << cfg->lx << " " << cfg->ly << " " << cfg->lz << std::endl;
  f << "Density " << density << std::endl;
  f << "Pressure parameters " << p0 << " " << p1 << " " << p2 << std::endl;
  f << "Thermostat " << thermostat << std::endl;
  f << "Temperature " << cfg->temperature << std::endl;
  f << "Cells properties " << std::endl;
  f << "Density " << std::endl;
  f << "Velocity" << std::endl;
  for (int64_t i = 0; i < nc; ++i) {
    f << density << std::endl;
    f << v[i] << " " << v[nc + i] << " " << v[2 * nc + i] << std::endl;
  }
  return f.good() ? FSL_OK : FSL_E_IO;
}

extern "C" int fsl_write_fluid_vtk(const char* path, int32_t mx, int32_t my, int32_t mz,
                                   const double* v) {
  if (!path || !v || mx < 1 || my < 1 || mz < 1) return FSL_E_ARG;
  FILE* fp = std::fopen(path, "w");
  if (!fp) return FSL_E_IO;
  VtkText t{fp};
  const int dims[3] = {mx + 1, my + 1, mz + 1};
  const int64_t nc = (int64_t)mx * my * mz;
  std::fprintf(fp, "# vtk DataFile Version 2.0\n");
  std::fprintf(fp, "Written using VisIt writer\n");
  std::fprintf(fp, "ASCII\n");
  std::fprintf(fp, "DATASET RECTILINEAR_GRID\n");
  std::fprintf(fp, "DIMENSIONS %d %d %d\n", dims[0], dims[1], dims[2]);
  const char* axis[3] = {"X", "Y", "Z"};
  for (int a = 0; a < 3; ++a) {
    if (a) t.section();
    std::fprintf(fp, "%s_COORDINATES %d double\n", axis[a], dims[a]);
    for (int i = 0; i < dims[a]; ++i) t.num((double)i);
  }
  t.section();
  std::fprintf(fp, "CELL_DATA %lld\n", (long long)nc);
  std::fprintf(fp, "VECTORS velocity double\n");
  // cell-centred velocity: the mean of the two faces of each cell along its
  // component (src/saveFluidVTK.cu:153-175)
  for (int64_t i = 0; i < nc; ++i) {
    const int x = (int)(i % mx), y = (int)((i / mx) % my), z = (int)(i / ((int64_t)mx * my));
    const int64_t ixm = (x == 0 ? mx - 1 : x - 1) + (int64_t)mx * (y + (int64_t)my * z);
    const int64_t iym = x + (int64_t)mx * ((y == 0 ? my - 1 : y - 1) + (int64_t)my * z);
    const int64_t izm = x + (int64_t)mx * (y + (int64_t)my * (z == 0 ? mz - 1 : z - 1));
    t.num(0.5 * (v[ixm] + v[i]));
    t.num(0.5 * (v[nc + iym] + v[nc + i]));
    t.num(0.5 * (v[2 * nc + izm] + v[2 * nc + i]));
  }
  t.end_line();
  t.end_line();
  const bool ok = std::ferror(fp) == 0;
  return (std::fclose(fp) == 0 && ok) ? FSL_OK : FSL_E_IO;
}
