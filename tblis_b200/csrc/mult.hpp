// mult.hpp -- contraction dispatch (tblis_tensor_mult and its extended form)
#pragma once

#include "common.hpp"

namespace tb
{

void mult_dispatch(const tblis_config* cfg,
                   const tblis_tensor* A, const label_type* idx_A,
                   const tblis_tensor* B, const label_type* idx_B,
                   tblis_tensor* C, const label_type* idx_C,
                   const tblis_b200_opts* opts, tblis_b200_report* report);

int device_sm_count();

} // namespace tb
