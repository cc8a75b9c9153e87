/* abi_ours.c -- compiles only when include/tblis_b200.h lays tblis_scalar and
 * tblis_tensor out as abi_layout.h states (dropin_c.c checks the same numbers
 * against TBLIS's own src/util/basic_types.h). */
#include <stddef.h>

#include "../../include/tblis_b200.h"
#include "abi_layout.h"

ABI_CHECK_LAYOUT(tblis_scalar, tblis_tensor);

int abi_ours_checked(void) { return 1; }
