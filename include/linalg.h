// Umbrella header of the C++ API: the LinAlgLib reference's public interface on
// the AMG-preconditioned Krylov path (library/include/linalg.h:193-239),
// implemented over the liblinalg_b200 C ABI (lab.h) with every computation on
// the GPU.
#ifndef LINALG_B200_LINALG_H
#define LINALG_B200_LINALG_H

#include "csr_matrix.h"
#include "vector.h"

#include "iterative_solvers/amg/amg.h"
#include "iterative_solvers/amg/amg_aggregation.h"
#include "iterative_solvers/amg/amg_strength.h"
#include "iterative_solvers/amg/amg_util.h"
#include "iterative_solvers/amg/rsamg.h"
#include "iterative_solvers/amg/saamg.h"
#include "iterative_solvers/amg/uaamg.h"
#include "iterative_solvers/iter_control.h"
#include "iterative_solvers/krylov/cg.h"
#include "iterative_solvers/krylov/gmres.h"
#include "iterative_solvers/preconditioner/preconditioner.h"
#include "linalg_math.h"

#endif
