// ConjugateGradient.h of the reference declares nothing; here it makes the CG solver
// (CGSolver.h) available to code that includes it.
#pragma once
#include "CGSolver.h"
