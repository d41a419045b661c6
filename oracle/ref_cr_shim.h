/* ORACLE — test infrastructure only.
 * Force-included (-include) when the reference host executor is compiled for
 * the correctly rounded comparison: every expf/logf call in the reference
 * sources resolves to the oracle's correctly rounded functions. */
#pragma once
#include <cmath>
extern "C" float or_cr_expf(float);
extern "C" float or_cr_logf(float);
#define expf or_cr_expf
#define logf or_cr_logf
