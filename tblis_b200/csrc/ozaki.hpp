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

// the same contraction in two phases, so a caller can queue the statistics
// of several contractions, do other work, and wait only for the statistics
struct OzakiJob
{
    GemmView v;
    const double* A = nullptr;
    const double* B = nullptr;
    double* C = nullptr;
    double alpha = 1, beta = 0, tol = 1e-12;
    int slices = 0;
    std::shared_ptr<GemmTables> tab;
    dbuf eA, eB, sA, sB;             // row exponents and sums of squares
    OzakiResult res;
};
// queues the row statistics of A and B on st
void ozaki_begin(OzakiJob& j, cudaStream_t st);
// picks the slice count (reads the statistics: stats_ready = they are
// complete, else this waits for st) and queues slicing and the INT8 GEMM
void ozaki_end(OzakiJob& j, cudaStream_t st, bool stats_ready);

} // namespace tb

namespace tb
{
// nonzero when an Ozaki kernel gave up a bounded wait (reads a device flag)
int ozaki_error_flag();
}
