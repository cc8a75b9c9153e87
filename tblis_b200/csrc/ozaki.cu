// ozaki.cu -- Ozaki split-precision contraction.
#include "ozaki.hpp"

namespace tb
{

OzakiResult ozaki_mult(const GemmView&, const double*, const double*, double*,
                       double, double, double, int, cudaStream_t)
{
    throw error(TB_ERR_ARG, "Ozaki method not built yet");
}

} // namespace tb
