// ozaki.hpp -- split-precision contraction on tcgen05: Ozaki INT8 or BF16
// slices, or a single TF32 / BF16 pass
#pragma once

#include "planner.hpp"

namespace tb
{

// element kind of the slice planes and of the tensor-core MMA
enum OzKind { OZ_I8 = 0, OZ_BF16 = 1, OZ_TF32 = 2 };

struct OzakiResult
{
    int scheme = 1;          // 1: slices (scheme I), 2: moduli (scheme II)
    int slices = 0;          // slice count, or the number of moduli for scheme II
    double est_error = 0;
};

// kind OZ_I8 / OZ_BF16 with single = false: Ozaki slices (slices = 0
// chooses the count from tol); single = true: one BF16 or TF32 pass.
// scheme (OZ_I8 only): 0 picks slices or moduli, whichever needs fewer INT8
// GEMMs for tol; 1 forces slices; 2 forces moduli (slices then counts the
// moduli, 0 = from tol)
OzakiResult ozaki_mult(const GemmView& v, const double* A, const double* B, double* C,
                       double alpha, double beta, double tol, int slices, cudaStream_t st,
                       int kind = OZ_I8, bool single = false, int scheme = 0);

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
    int kind = OZ_I8;
    bool single = false;
    int scheme = 0;
    std::shared_ptr<GemmTables> tab;
    dbuf eA, eB, sA, sB;             // row exponents and sums of squares
    OzakiResult res;
};
// queues the row statistics of A and B on st
void ozaki_begin(OzakiJob& j, cudaStream_t st);
// picks the slice count (reads the statistics: stats_ready = they are
// complete, else this waits for st) and queues slicing and the slice GEMM
void ozaki_end(OzakiJob& j, cudaStream_t st, bool stats_ready);

} // namespace tb

namespace tb
{
// nonzero when an Ozaki kernel gave up a bounded wait since the last check
// (reads and clears a device flag)
int ozaki_error_flag();
// test support: the Ozaki GEMM kernels skip the copies of k step (moduli
// kernel: stage) `step` (-1: none) and bound every wait by wait_seconds (<= 0:
// the default 2 s)
void ozaki_inject_wait_timeout(int step, double wait_seconds);
}
