// Stand-in for the reference's Metropolis generator (src/Apps/gaugefieldfactory.cpp),
// which does not compile against the reference's own headers (GluonField has no
// setToUnity, no operator()(x,y,z,t)).  It lets the reference's FLOW application
// (LatticeQCDMain + JSON layer + WilsonFlow + I/O) link into oracle/_ref/lattice_qcd;
// asking that binary for "PGFG" reports the stand-in and exits.  Test infrastructure.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "Apps/gaugefieldfactory.h"

GaugeFieldFactory::GaugeFieldFactory(int, int, int, double, std::string) {}
void GaugeFieldFactory::execute() {
    std::fprintf(stderr, "PGFG is not available in this build of the reference (its source does not compile)\n");
    std::exit(2);
}
