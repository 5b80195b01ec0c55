/*
 * The reference objects a checker run built (oracle/ref_harness.cc): test
 * infrastructure, for harnesses that construct reference-side classes from
 * the same parsed script (oracle/dropin_harness.cc).
 */
#ifndef SHHD_REF_HARNESS_H
#define SHHD_REF_HARNESS_H

#include "domain.h"
#include "model_free_energy.h"
#include "model_thermodynamics.h"
#include "model_transport_coefficient.h"
#include "simulationinfo.h"
#include "state.h"

struct RefRunView {
    const Params* params;
    const Domain2D* domain;
    const Thermodynamics* thermodynamics;
    const FreeEnergy* free_energy;
    const TransportCoefficient* transport;
    State* state;   // the script's initial state, as Project::apply_initial_conditions leaves it
};

// the objects of a run made by shref_create (false for a null handle)
bool shref_view(void* handle, RefRunView& out);

#endif
