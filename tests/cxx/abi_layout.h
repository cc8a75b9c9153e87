/* abi_layout.h -- the byte layout both TBLIS's src/util/basic_types.h
 * (tblis_scalar :154-175, tblis_tensor :471-479) and this library's
 * include/tblis_b200.h must have: the drop-in programs static_assert these
 * numbers against TBLIS's own header, abi_ours.c against this library's. */
#ifndef TBLIS_B200_TEST_ABI_LAYOUT_H
#define TBLIS_B200_TEST_ABI_LAYOUT_H

#define ABI_SCALAR_SIZE        24
#define ABI_SCALAR_OFF_DATA     0
#define ABI_SCALAR_OFF_TYPE    16
#define ABI_TENSOR_SIZE        64
#define ABI_TENSOR_OFF_TYPE     0
#define ABI_TENSOR_OFF_CONJ     4
#define ABI_TENSOR_OFF_SCALAR   8
#define ABI_TENSOR_OFF_DATA    32
#define ABI_TENSOR_OFF_NDIM    40
#define ABI_TENSOR_OFF_LEN     48
#define ABI_TENSOR_OFF_STRIDE  56

#define ABI_CHECK_LAYOUT(SCALAR, TENSOR)                                                           \
    _Static_assert(sizeof(SCALAR) == ABI_SCALAR_SIZE, "tblis_scalar size");                        \
    _Static_assert(offsetof(SCALAR, data) == ABI_SCALAR_OFF_DATA, "tblis_scalar.data");            \
    _Static_assert(offsetof(SCALAR, type) == ABI_SCALAR_OFF_TYPE, "tblis_scalar.type");            \
    _Static_assert(sizeof(TENSOR) == ABI_TENSOR_SIZE, "tblis_tensor size");                        \
    _Static_assert(offsetof(TENSOR, type) == ABI_TENSOR_OFF_TYPE, "tblis_tensor.type");            \
    _Static_assert(offsetof(TENSOR, conj) == ABI_TENSOR_OFF_CONJ, "tblis_tensor.conj");            \
    _Static_assert(offsetof(TENSOR, scalar) == ABI_TENSOR_OFF_SCALAR, "tblis_tensor.scalar");      \
    _Static_assert(offsetof(TENSOR, data) == ABI_TENSOR_OFF_DATA, "tblis_tensor.data");            \
    _Static_assert(offsetof(TENSOR, ndim) == ABI_TENSOR_OFF_NDIM, "tblis_tensor.ndim");            \
    _Static_assert(offsetof(TENSOR, len) == ABI_TENSOR_OFF_LEN, "tblis_tensor.len");               \
    _Static_assert(offsetof(TENSOR, stride) == ABI_TENSOR_OFF_STRIDE, "tblis_tensor.stride")

#endif
