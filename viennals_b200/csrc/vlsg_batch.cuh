// vlsg_batch.cuh -- the per-domain time bookkeeping of the batching form.
//
// The batching form advances many independent domains in one brick box (the
// domain table of GridDev): every band pass, rate pass and value update is
// one launch over the bricks of all domains.  What differs per domain is the
// time step: the rate pass leaves per domain its smallest per-point step and
// its Lax-Friedrichs alphas (RED_* words), and kDomainSteps turns them into
// the domain's stage step with the rule computeRates applies to a single
// domain (lsAdvect.hpp:595-611 plus the Lax-Friedrichs bound of
// reduceTimeStepHamiltonJacobi): min(cap, smallest step, 1 / sum_k
// alpha_k / gridDelta).  The steps stay on the device; the value update reads
// them per slot.  kDomainTime combines the stage steps into each domain's
// advected time as the integration schemes do
// (lsAdvectIntegrationSchemes.hpp:46-168).
#pragma once

#include "vlsg_common.cuh"
#include "vlsg_rates.cuh"

namespace vlsg {
namespace { // internal linkage: every compilation unit has its own copy

// Per-domain step of a stage.  cap: the stage's maximum step per domain
// (null: none); out: the step; red: the rate pass's RED_* words, reset here
// for the next pass; updates: point updates so far (active points of every
// stage).  A domain whose first stage gets no positive step sets err bit 512
// (`first`): the reference then stops that domain's RK step, which the one
// shared stage sequence cannot do.
__global__ void kDomainSteps(int nDom, unsigned long long *red, const double *delta,
                             int lfFamily, const double *cap, double *out,
                             unsigned long long *updates, int first, int *err) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nDom; d += gridDim.x * blockDim.x) {
    unsigned long long *r = red + (size_t)RED_WORDS * d;
    const double maxTimeStep = cap ? cap[d] : DBL_MAX;
    double tempMax = maxTimeStep;
    double m = DBL_MAX; // no active point: no bound from the points
    if (r[RED_MIN] != ~0ull) m = __longlong_as_double((long long)r[RED_MIN]);
    if (m < tempMax) tempMax = m;
    if (lfFamily) {
      double timeStep = 0;
      for (int i = 0; i < 3; ++i)
        timeStep += __longlong_as_double((long long)r[RED_ALPHA + i]) / delta[d];
      timeStep = 1.0 / timeStep;
      tempMax = (tempMax < timeStep) ? tempMax : timeStep;
    }
    const double dt = tempMax < maxTimeStep ? tempMax : maxTimeStep;
    out[d] = dt;
    if (first && !(dt > 0.)) atomicOr(err, 512);
    updates[d] += r[RED_ACTIVE];
    r[RED_MIN] = ~0ull;
    r[RED_ALPHA] = r[RED_ALPHA + 1] = r[RED_ALPHA + 2] = 0ull;
    r[RED_ACTIVE] = 0ull;
  }
}

// Advected time of the step per domain from its stage steps a, b, c:
// forward Euler a, Heun (a + b) / 2, SSP RK3 (a + b + 4 c) / 6.
__global__ void kDomainTime(int nDom, int temporal, const double *a, const double *b,
                            const double *c, double *time) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nDom; d += gridDim.x * blockDim.x) {
    if (temporal == VLSG_RUNGE_KUTTA_2ND_ORDER) time[d] = 0.5 * a[d] + 0.5 * b[d];
    else if (temporal == VLSG_RUNGE_KUTTA_3RD_ORDER) time[d] = (a[d] + b[d] + 4.0 * c[d]) / 6.0;
    else time[d] = a[d];
  }
}

} // namespace
} // namespace vlsg
