// ref_stubs.cpp -- link stubs for the parts of fluam that the host build of
// the stokesLimit path does not compile.  TEST INFRASTRUCTURE ONLY.
//
// src/main.cpp dispatches to every scheme of fluam; only schemeStokesLimit is
// built, the others report that they are not built and fail.  The end of
// schemeStokesLimit frees the host cell arrays through
// freeMemoryQuasiNeutrallyBuoyant (src/schemeQuasiNeutrallyBuoyant.cu:98-110);
// that release is done here.
#include <iostream>

#include "header.h"
#include "cells.h"

namespace {
bool not_built(const char* what) {
  std::cout << "REFERENCE HOST BUILD: " << what << " is not built" << std::endl;
  return 0;
}
}  // namespace

bool freeMemoryQuasiNeutrallyBuoyant() {
  delete[] cvx;
  delete[] cvy;
  delete[] cvz;
  delete[] crx;
  delete[] cry;
  delete[] crz;
  delete[] cDensity;
  std::cout << "FREE MEMORY :                   DONE" << std::endl;
  return 1;
}

// The reference's freeBondedForces (src/initializeBondedForces.cpp:186-207)
// releases host arrays and falls off the end of a bool function; the host
// build renames it and calls this one instead (the arrays die with the
// process).
bool freeBondedForces() { return 1; }

bool createBoundaries() { return not_built("boundary (fileboundary) input"); }
bool freeBoundaries() { return 1; }

#define FLUAM_SCHEME_STUB(name) \
  bool name() { return not_built(#name); }
FLUAM_SCHEME_STUB(schemeBinaryMixture)
FLUAM_SCHEME_STUB(schemeBinaryMixtureWall)
FLUAM_SCHEME_STUB(schemeBoundary)
FLUAM_SCHEME_STUB(schemeCompressibleParticles)
FLUAM_SCHEME_STUB(schemeContinuousGradient)
FLUAM_SCHEME_STUB(schemeFreeEnergyCompressibleParticles)
FLUAM_SCHEME_STUB(schemeGiantFluctuations)
FLUAM_SCHEME_STUB(schemeIncompressibleBinaryMixture)
FLUAM_SCHEME_STUB(schemeIncompressibleBinaryMixtureMidPoint)
FLUAM_SCHEME_STUB(schemeIncompressibleBoundary)
FLUAM_SCHEME_STUB(schemeMomentumCoupling)
FLUAM_SCHEME_STUB(schemeParticlesWall)
FLUAM_SCHEME_STUB(schemeQuasiNeutrallyBuoyant)
FLUAM_SCHEME_STUB(schemeQuasiNeutrallyBuoyant2D)
FLUAM_SCHEME_STUB(schemeQuasiNeutrallyBuoyant4pt2D)
FLUAM_SCHEME_STUB(schemeRK3)
FLUAM_SCHEME_STUB(schemeRK3Ghost)
FLUAM_SCHEME_STUB(schemeSemiImplicitCompressibleParticles)
FLUAM_SCHEME_STUB(schemeThermostat)
