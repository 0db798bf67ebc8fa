// Drop-in ADER time stepper: the interface of the reference's Temporal_ader.h
// (mrnorman/awflCloud Temporal_ader.h:1-83) over the B200 spatial operator.
//
// timeStep() runs the three directional splits (Temporal_ader.h:48-72); each split is the
// spatial operator's computeTendencies followed by the apply, executed as one fused kernel
// (Spatial::computeAndApplyTendencies), which gives the same results as the two calls.
// Tracers are left unchanged, as the reference's are (it compiles their transport out),
// unless the YAML key tracer_transport is true: then each split advances them first.
#pragma once

#include "const.h"

int constexpr nTimeDerivs = 1;
bool constexpr timeAvg = true;
int constexpr nAder = ngll;

template <class Spatial> class Temporal_ader {
 public:
  static_assert(nTimeDerivs <= ngll, "ERROR: nTimeDerivs must be <= ngll.");

  typedef typename Spatial::StateTendArr StateTendArr;
  typedef typename Spatial::StateArr StateArr;
  typedef typename Spatial::TracerTendArr TracerTendArr;
  typedef typename Spatial::TracerArr TracerArr;
  typedef typename Spatial::Location Location;

  StateTendArr stateTendArr;
  TracerTendArr tracerTendArr;

  Spatial spaceOp;

  void init(std::string inFile) {
    spaceOp.init(inFile);
    stateTendArr = spaceOp.createStateTendArr();
    tracerTendArr = spaceOp.createTracerTendArr();
  }

  void timeStep(StateArr &stateArr, TracerArr &tracerArr, real dt) {
    for (int spl = 0; spl < spaceOp.numSplit(); spl++) {
      spaceOp.computeAndApplyTendencies(stateArr, tracerArr, dt, spl);
    }
  }

  void finalize(StateArr &state, TracerArr &tracers) { spaceOp.finalize(state, tracers); }

  const char *getTemporalName() { return "ADER-DT"; }
};
