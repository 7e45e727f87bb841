/* project-written GSL API stand-in for compiling the oracle; see gsl_shim_all.h */
#pragma once
#include "gsl_shim_all.h"
