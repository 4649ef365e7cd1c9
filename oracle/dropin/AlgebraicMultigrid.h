// Stand-in for Smoke_Solver/AlgebraicMultigrid.h in the drop-in build of the
// reference (oracle/build_ref.py, libvflip_ref_dropin.so).  TEST
// INFRASTRUCTURE ONLY.
//
// The reference's translation units reach their solver through this header
// (Smoke_solver3D.h:21, sub_domain.h:19).  This version keeps the includes and
// using-directives those units receive from the original, and takes
// ivock::AMGPCGSolve from include/vflip/amgpcg_dropin.hpp - the GPU solve
// through vflip_amgpcg_solve_csr - instead of the CPU multigrid, so
// SmokeSolver3D::pcg_projection (Smoke_solver3D.cpp:1120) and
// SubDomainSolver::pcg_projection (sub_domain.cpp:739) run unchanged on the GPU.
#ifndef _AMG_H_
#define _AMG_H_

#include <cmath>
#include <iostream>
#include <vector>

#include "GeometricLevelGen.h"
#include "blas_wrapper.h"
#include "pcg_solver.h"
#include "sparse_matrix.h"
#include "tbb/tbb.h"
#include "util.h"
#include "vec.h"

using namespace std;
using namespace BLAS;

#include "vflip/amgpcg_dropin.hpp"

#endif
