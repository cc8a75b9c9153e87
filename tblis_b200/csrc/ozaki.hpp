// ozaki.hpp -- Ozaki split-precision contraction (INT8 slices on tcgen05)
#pragma once

#include "planner.hpp"

namespace tb
{

struct OzakiResult
{
    int slices = 0;
    double est_error = 0;
};

OzakiResult ozaki_mult(const GemmView& v, const double* A, const double* B, double* C,
                       double alpha, double beta, double tol, int slices, cudaStream_t st);

} // namespace tb

namespace tb
{
// nonzero when an Ozaki kernel gave up a bounded wait (reads a device flag)
int ozaki_error_flag();
}
