// Link stubs for the reference base classes of MesonCorrelator, ChiralCondensate, OutputSweep
// and ReadStartGaugeConfiguration that the harness never needs as a program: LatticeSweep and
// StartGaugeConfiguration, whose factories pull in every sweep and starter of the program.
// TEST INFRASTRUCTURE ONLY (oracle/build_ref.sh).
#include <cstdlib>
#include <iostream>

#include "LatticeSweep.h"
#include "starters/StartGaugeConfiguration.h"

namespace Update {

LatticeSweep::LatticeSweep() : numberTimes(1), sweepToJump(1) {}
LatticeSweep::~LatticeSweep() {}

// the base of ReadStartGaugeConfiguration (its factory, in StartGaugeConfiguration.cpp, pulls
// in every starter)
StartGaugeConfiguration::StartGaugeConfiguration() : LatticeSweep() {}
StartGaugeConfiguration::~StartGaugeConfiguration() {}

}  // namespace Update
