// Include-path stand-in for the numerics library header linear/solvers/preconditioner.hpp that MarkovKit's programs include:
// num::idx, num::vec, num::gmres, num::jacobi_preconditioner and num::ilu0_preconditioner are
// declared by the facade, so a program written against the reference builds with -I include/mk.
#pragma once

#include "../../markovkit.hpp"
