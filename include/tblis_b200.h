/*
 * tblis_b200.h -- public C ABI of the B200 (sm_100a) TBLIS drop-in.
 *
 * The first part re-declares TBLIS's own C ABI with byte-identical types, so
 * a program built against TBLIS's headers (src/tblis.h) links against
 * libtblis_b200.so instead of libtblis.so unchanged. Each declaration cites
 * the reference interface it replaces (paths relative to the TBLIS tree).
 *
 * Data residency: tensor data may live in device memory (cudaMalloc'd or
 * managed; the call is stream-ordered on the library stream and returns
 * without waiting, except dot/reduce which return a host scalar and so
 * synchronise) or in host memory (the call stages the touched extent to the
 * device and back and returns when the result is in host memory). No call
 * computes on the CPU.
 *
 * Errors: the TBLIS entry points return void like the reference. A failure
 * (unsupported type, malformed labels, CUDA error, no device) records a
 * thread-local error readable with tblis_b200_last_error(); with the
 * environment variable TBLIS_B200_ABORT_ON_ERROR=1 it aborts, like the
 * reference's TBLIS_ASSERT in debug builds (src/util/basic_types.h:612-621).
 */
#ifndef TBLIS_B200_H
#define TBLIS_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- types (src/util/basic_types.h) ------------------------------------ */

typedef ptrdiff_t len_type;     /* configure.ac:91-101 default */
typedef ptrdiff_t stride_type;  /* configure.ac:103-113 default */
typedef char label_type;        /* configure.ac:115-123 default */

/* src/util/basic_types.h:53-64 */
typedef enum
{
    REDUCE_SUM      = 0,
    REDUCE_SUM_ABS  = 1,
    REDUCE_MAX      = 2,
    REDUCE_MAX_ABS  = 3,
    REDUCE_MIN      = 4,
    REDUCE_MIN_ABS  = 5,
    REDUCE_NORM_1   = REDUCE_SUM_ABS,
    REDUCE_NORM_2   = 6,
    REDUCE_NORM_INF = REDUCE_MAX_ABS
} reduce_t;

/* src/util/basic_types.h:66-73 */
typedef enum
{
    TYPE_SINGLE   = 0,
    TYPE_FLOAT    = TYPE_SINGLE,
    TYPE_DOUBLE   = 1,
    TYPE_SCOMPLEX = 2,
    TYPE_DCOMPLEX = 3
} type_t;

/* src/util/basic_types.h:154-175: 16-byte value union + type tag (24 bytes) */
typedef struct tblis_scalar
{
    union
    {
        float s;
        double d;
        float c[2];
        double z[2];
    } data;
    type_t type;
} tblis_scalar;

/* src/util/basic_types.h:471-479 (64 bytes) */
typedef struct tblis_tensor
{
    type_t type;
    int conj;
    tblis_scalar scalar;
    void* data;
    unsigned ndim;
    len_type* len;
    stride_type* stride;
} tblis_tensor;

/* src/util/thread.h:13 (tci_comm) and src/util/basic_types.h:51: opaque here.
 * A non-null comm means the caller is inside a TCI parallel region; only its
 * master thread may call this library (the GPU is driven by one host thread). */
typedef struct tci_comm tblis_comm;
typedef struct tblis_config_s tblis_config;

/* ---- reference C ABI ---------------------------------------------------- */

/* src/iface/3t/mult.h:17-20, src/iface/3t/mult.cxx:24-165 */
void tblis_tensor_mult(const tblis_comm* comm, const tblis_config* cfg,
                       const tblis_tensor* A, const label_type* idx_A,
                       const tblis_tensor* B, const label_type* idx_B,
                             tblis_tensor* C, const label_type* idx_C);

/* src/iface/1t/add.h:17-19, src/iface/1t/add.cxx:24-110 */
void tblis_tensor_add(const tblis_comm* comm, const tblis_config* cfg,
                      const tblis_tensor* A, const label_type* idx_A,
                            tblis_tensor* B, const label_type* idx_B);

/* src/iface/1t/dot.h:17-20, src/iface/1t/dot.cxx:16-74 */
void tblis_tensor_dot(const tblis_comm* comm, const tblis_config* cfg,
                      const tblis_tensor* A, const label_type* idx_A,
                      const tblis_tensor* B, const label_type* idx_B,
                      tblis_scalar* result);

/* src/iface/1t/reduce.h:17-19, src/iface/1t/reduce.cxx:16-68 */
void tblis_tensor_reduce(const tblis_comm* comm, const tblis_config* cfg, reduce_t op,
                         const tblis_tensor* A, const label_type* idx_A,
                         tblis_scalar* result, len_type* idx);

/* src/iface/1t/scale.h:17-18, src/iface/1t/scale.cxx:20-60 */
void tblis_tensor_scale(const tblis_comm* comm, const tblis_config* cfg,
                        tblis_tensor* A, const label_type* idx_A);

/* src/iface/1t/set.h:17-18, src/iface/1t/set.cxx:16-50 */
void tblis_tensor_set(const tblis_comm* comm, const tblis_config* cfg,
                      const tblis_scalar* alpha, tblis_tensor* A, const label_type* idx_A);

/* src/iface/1t/shift.h:17-18, src/iface/1t/shift.cxx:14-75 */
void tblis_tensor_shift(const tblis_comm* comm, const tblis_config* cfg,
                        const tblis_scalar* alpha, tblis_tensor* A, const label_type* idx_A);

/* src/util/basic_types.h:549-579, defs src/util/basic_types.cxx:197-247 */
void tblis_init_scalar_s(tblis_scalar* s, float value);
void tblis_init_scalar_d(tblis_scalar* s, double value);
void tblis_init_tensor_scaled_s(tblis_tensor* t, float scalar, unsigned ndim,
                                len_type* len, float* data, stride_type* stride);
void tblis_init_tensor_scaled_d(tblis_tensor* t, double scalar, unsigned ndim,
                                len_type* len, double* data, stride_type* stride);
void tblis_init_tensor_s(tblis_tensor* t, unsigned ndim, len_type* len, float* data,
                         stride_type* stride);
void tblis_init_tensor_d(tblis_tensor* t, unsigned ndim, len_type* len, double* data,
                         stride_type* stride);

/* src/util/thread.h:21-23, src/util/thread.cxx:108-118: kept for source
 * compatibility; the value is recorded and returned but the GPU path does not
 * use CPU threads. */
unsigned tblis_get_num_threads(void);
void tblis_set_num_threads(unsigned num_threads);

/* src/util/configs.h:11: returns a GPU configuration by name, or NULL.
 * Names: "b200_fp64" (default; FP64 DMMA), "b200_ozaki_i8" (Ozaki INT8 on
 * tcgen05: slices or moduli, whichever needs less INT8 work for the
 * tolerance), "b200_ozaki_bf16" (Ozaki BF16 slices), "b200_ozaki_crt" (Ozaki
 * INT8 over pairwise-coprime moduli only, scheme II), "b200_tf32" and
 * "b200_bf16" (one low-precision pass with FP32 accumulation). */
const tblis_config* tblis_get_config(const char* name);

/* ---- extensions (no counterpart in the reference) ------------------------ */

/* Last error of the calling thread: 0 = none. The message is kept until the
 * next failing call; tblis_b200_clear_error() resets it. */
int tblis_b200_last_error(void);
const char* tblis_b200_last_error_string(void);
void tblis_b200_clear_error(void);

/* Stream (a cudaStream_t) that subsequent calls of this host thread enqueue
 * on; NULL = the legacy default stream. */
void tblis_b200_set_stream(void* stream);
void* tblis_b200_get_stream(void);
/* Waits for all work this library enqueued on the current stream. Records
 * TB_ERR_TIMEOUT (6) as the last error when an Ozaki kernel or the packed
 * grouped FP64 kernel gave up one of its bounded waits since the previous
 * check (the flag is then cleared). */
void tblis_b200_synchronize(void);

/* Test support for the failure detection of the Ozaki kernels (no reference
 * counterpart): the INT8/BF16 slice GEMM and the moduli GEMM skip the operand
 * copies of k step (moduli kernel: pipeline stage) `step`, so the wait for it
 * runs out after wait_seconds instead of the default 2 s; the kernel then
 * records the timeout, drains its copies in flight, frees its tensor memory
 * and returns, and tblis_b200_synchronize reports it. step = -1 and
 * wait_seconds <= 0 restore normal operation. Returns 0 or an error code. */
int tblis_b200_ozaki_inject_wait_timeout(int step, double wait_seconds);

/* The same for the packed grouped FP64 GEMM (DPD, indexed DPD and batches on
 * the packed path; no reference counterpart): its producer issues no copy for
 * the CTA's pipeline stage `step`, and every bounded wait gives up after
 * wait_seconds; the kernel records the timeout, waits for the copies it
 * issued and returns. step = -1 and wait_seconds <= 0 restore normal
 * operation. Returns 0 or an error code. */
int tblis_b200_grouped_inject_wait_timeout(int step, double wait_seconds);

/* Normwise relative tolerance carried by a configuration (used by the Ozaki
 * configurations to pick the slice count; 0 restores the default 1e-12). */
void tblis_b200_config_set_tolerance(tblis_config* cfg, double tol);
double tblis_b200_config_get_tolerance(const tblis_config* cfg);

/* Per-call options and report of the extended contraction entry point. */
typedef struct tblis_b200_opts
{
    int method;          /* 0 = from cfg, 1 = FP64 DMMA, 2 = Ozaki INT8 (slices
                            or moduli, whichever needs less INT8 work for the
                            tolerance), 3 = Ozaki BF16 slices, 4 = one TF32
                            pass, 5 = one BF16 pass (FP32 accumulation; no
                            tolerance), 6 = Ozaki INT8 over moduli (scheme II) */
    int slices;          /* Ozaki slice count (method 2: forces slices) or
                            moduli count (method 6, 2..16); 0 = from tolerance */
    double tolerance;    /* normwise relative target; 0 = from cfg */
} tblis_b200_opts;

typedef struct tblis_b200_report
{
    int method;          /* method that ran (6 when method 2 chose moduli) */
    int slices;          /* slice count, or moduli count for method 6 (0 for FP64) */
    double est_error;    /* a-priori normwise error estimate */
    double flops;        /* algorithmic FLOPs, 2*m*n*k*l */
    int64_t m, n, k, l;  /* GEMM view of the contraction */
    int kernels;         /* kernels launched by this call */
} tblis_b200_report;

/* tblis_tensor_mult with explicit method/tolerance and a report; returns 0
 * on success, else an error code (also recorded as the last error). */
int tblis_b200_tensor_mult_ex(const tblis_config* cfg,
                              const tblis_tensor* A, const label_type* idx_A,
                              const tblis_tensor* B, const label_type* idx_B,
                                    tblis_tensor* C, const label_type* idx_C,
                              const tblis_b200_opts* opts, tblis_b200_report* report);

/* The product's block-scatter vector builder (restating
 * src/matrix/block_scatter_matrix.hpp:249-258 for double), exported so the
 * tests can compare it bit for bit with the reference. */
void tblis_b200_fill_block_scatter(unsigned ndim, const len_type* len,
                                   const stride_type* stride, len_type BS,
                                   stride_type off, stride_type size,
                                   stride_type* scat, stride_type* bs, int pack_3d);

/* The product's index-group split of a contraction (src/iface/3t/mult.cxx:30-116
 * and src/internal/3t/dense/mult.cxx:214-263), as label strings per group in
 * their GEMM order and m/n/k/l. Returns 0 or an error code. */
int tblis_b200_mult_groups(const tblis_tensor* A, const label_type* idx_A,
                           const tblis_tensor* B, const label_type* idx_B,
                           const tblis_tensor* C, const label_type* idx_C,
                           char* idx_AB, char* idx_AC, char* idx_BC, char* idx_ABC,
                           int64_t* mnkl);

/* Number of kernels this library launched since the process started. */
int64_t tblis_b200_kernel_count(void);

/* Per-kernel device timing (no reference counterpart). While enabled, the
 * library brackets each launch of its contraction and transpose kernels
 * (gemm_f64_kernel, gemm_f64_grouped_kernel, ozaki_gemm_kernel, oz_stats,
 * oz_slice, oz_crt_gemm, oz_crt_combine, k_transpose, k_add_rows) with a
 * CUDA event pair on the launching stream. Enabling or
 * disabling clears the records; reading waits for the recorded launches and
 * returns their summed device time and count for one kernel name. */
int tblis_b200_kernel_timer(int enable);
int tblis_b200_kernel_timer_read(const char* kernel, double* total_ms, int64_t* launches);

/* ---- DPD (irrep block-sparse) tensors ------------------------------------ */

/* A dense-stored DPD tensor as MArray's dpd_varray lays it out
 * (src/external/marray/include/dpd_varray_base.hpp:10-128,
 * dpd_marray_base.hpp:34-228): the symmetry-allowed blocks of irrep `irrep`
 * (XOR of the block's irreps) stored back to back in one buffer of
 * tblis_b200_dpd_size() elements. len is [ndim][nirrep] row-major; layout is
 * MArray's dpd_layout type (0 BALANCED_COLUMN_MAJOR, 1 BALANCED_ROW_MAJOR,
 * 2 BLOCKED_COLUMN_MAJOR, 3 BLOCKED_ROW_MAJOR, 4 PREFIX_COLUMN_MAJOR,
 * 5 PREFIX_ROW_MAJOR; -1 = MArray's default, PREFIX_ROW_MAJOR). */
typedef struct tblis_b200_dpd_tensor
{
    type_t type;
    int conj;
    tblis_scalar scalar;
    void* data;
    unsigned ndim;
    unsigned nirrep;
    unsigned irrep;
    const len_type* len;
    int layout;
} tblis_b200_dpd_tensor;

/* C = alpha*A*B + beta*C over DPD tensors (alpha = A.scalar*B.scalar, beta =
 * C.scalar), the C entry of tblis::mult over dpd_varray_view
 * (src/iface/3t/mult.cxx:170-289, src/internal/3t/dpd/mult.cxx:223-356): one
 * GEMM per irrep of the contracted labels, all in one grouped launch. Labels
 * must be unique per tensor; labels shared by all three tensors (batch
 * labels) are supported as in src/internal/3t/dpd/mult.cxx:1082-1115.
 * Returns 0 or an error code. report->m = irrep GEMMs launched, report->n =
 * tile configuration picked by the autotuner. */
int tblis_b200_dpd_mult(const tblis_b200_dpd_tensor* A, const label_type* idx_A,
                        const tblis_b200_dpd_tensor* B, const label_type* idx_B,
                              tblis_b200_dpd_tensor* C, const label_type* idx_C,
                        tblis_b200_report* report);

/* A DPD tensor given by the geometry of its stored blocks rather than by one
 * of MArray's storage layouts: what a dpd_varray_view reports for each block
 * through operator()(irreps) (dpd_varray_base.hpp:482-508), which also covers
 * permuted views. len is [ndim][nirrep]; offset[t] and stride[t*ndim + d]
 * describe the block whose irreps are (i_0, ..., i_{ndim-1}) at
 * t = sum_d i_d*nirrep^d (dimension 0 fastest); offset -1 marks tuples that
 * are not stored. Offsets and strides are in elements, non-negative. */
typedef struct tblis_b200_dpd_block_table
{
    type_t type;
    int conj;
    tblis_scalar scalar;
    void* data;
    unsigned ndim;
    unsigned nirrep;
    unsigned irrep;
    const len_type* len;
    const stride_type* offset;
    const stride_type* stride;
} tblis_b200_dpd_block_table;

/* tblis_b200_dpd_mult over block tables: the entry the C++ overload
 * tblis::mult(comm, alpha, dpd_varray_view<const T> A, ...) of
 * src/iface/3t/mult.h:56-60 reaches (libtblis_b200_cxx.so). */
int tblis_b200_dpd_mult_blocks(const tblis_b200_dpd_block_table* A, const label_type* idx_A,
                               const tblis_b200_dpd_block_table* B, const label_type* idx_B,
                                     tblis_b200_dpd_block_table* C, const label_type* idx_C,
                               tblis_b200_report* report);

/* Level-1 operations over DPD tensors given by block tables: the C entries
 * of tblis::add / dot / reduce / scale / set / shift over dpd_varray_view
 * (src/iface/1t/{add,dot,reduce,scale,set,shift}.cxx). add: B = alpha*A +
 * beta*B (alpha = A.scalar, beta = B.scalar) with A-only labels traced and
 * B-only labels replicated per block; dot: alpha_A*alpha_B*sum A*B over the
 * blocks (labels must match); reduce: reduce_t over every stored element,
 * idx = the element's offset from data; scale: A *= A.scalar; set: A =
 * alpha; shift: A = alpha + A.scalar*A. Each runs the dense kernel of the
 * operation on every stored block in place. Return 0 or an error code. */
int tblis_b200_dpd_add(const tblis_b200_dpd_block_table* A, const label_type* idx_A,
                       tblis_b200_dpd_block_table* B, const label_type* idx_B);
int tblis_b200_dpd_dot(const tblis_b200_dpd_block_table* A, const label_type* idx_A,
                       const tblis_b200_dpd_block_table* B, const label_type* idx_B, tblis_scalar* result);
int tblis_b200_dpd_reduce(reduce_t op, const tblis_b200_dpd_block_table* A, const label_type* idx_A,
                          tblis_scalar* result, len_type* idx);
int tblis_b200_dpd_scale(tblis_b200_dpd_block_table* A, const label_type* idx_A);
int tblis_b200_dpd_set(const tblis_scalar* alpha, tblis_b200_dpd_block_table* A, const label_type* idx_A);
int tblis_b200_dpd_shift(const tblis_scalar* alpha, tblis_b200_dpd_block_table* A, const label_type* idx_A);

/* The dense form of a DPD tensor (block_to_full,
 * src/internal/1t/dpd/util.hpp:70-102): dimension d of the dense tensor F
 * has the sum over irreps of A's lengths of dimension d, irrep x occupying
 * the range after the lengths of the irreps below x. F (any strides, A's
 * element type) is set to zero, then every stored block of A is copied into
 * its region. Scalars and conjugation flags do not apply. Returns 0 or an
 * error code. */
int tblis_b200_dpd_block_to_full(const tblis_b200_dpd_block_table* A, tblis_tensor* F);

/* The reverse (full_to_block, src/internal/1t/dpd/util.hpp:104-133): every
 * stored block of A gets a copy of its region of the dense tensor F; storage
 * of A outside its blocks is left as it is. Returns 0 or an error code. */
int tblis_b200_dpd_full_to_block(const tblis_tensor* F, tblis_b200_dpd_block_table* A);

/* An indexed DPD tensor as MArray's indexed_dpd_varray holds it
 * (indexed_dpd_varray_base.hpp, indexed_dpd_varray.hpp:309-370): the first
 * dense_ndim dimensions are DPD dimensions; each of the other (indexed)
 * dimensions has one fixed irrep, and the tensor stores nidx entries, each a
 * DPD tensor over the dense dimensions (irrep dense_irrep) at data[i] with an
 * index tuple indices[i][...] and a scalar factor[i] (NULL = all 1). len is
 * [ndim][nirrep]; the dense blocks of every entry share one block table
 * (offset/stride relative to the entry's data, as tblis_b200_dpd_block_table). */
typedef struct tblis_b200_indexed_dpd_tensor
{
    type_t type;
    tblis_scalar scalar;
    unsigned ndim;
    unsigned dense_ndim;
    unsigned nirrep;
    unsigned dense_irrep;
    const len_type* len;
    const unsigned* idx_irrep;
    len_type nidx;
    const len_type* indices;
    void* const* data;          /* per entry: its dense storage (elements of `type`) */
    const void* factor;         /* per entry: its factor (an element of `type`), or NULL for 1 */
    const stride_type* offset;
    const stride_type* stride;
} tblis_b200_indexed_dpd_tensor;

/* C = alpha*A*B + beta*C over indexed DPD tensors (alpha = A.scalar*B.scalar,
 * beta = C.scalar), the entry of tblis::mult over indexed_dpd_varray_view
 * (src/iface/3t/mult.cxx:412-533): C entry i is first scaled by f_C[i]*beta
 * (beta == 1: untouched; beta == 0 or f_C[i] == 0: zeroed), then it
 * receives alpha*f_C[i]*f_A[j]*f_B[k]*(A_j . B_k) from every pair of
 * A and B entries whose index values agree with it and with each other; a
 * label indexed in one tensor and dense in another selects that slice. Each
 * consistent triple runs as one grouped launch of the FP64 kernel. Labels
 * dense in all three tensors are not supported. report->m = triples launched.
 * Returns 0 or an error code. */
int tblis_b200_indexed_dpd_mult(const tblis_b200_indexed_dpd_tensor* A, const label_type* idx_A,
                                const tblis_b200_indexed_dpd_tensor* B, const label_type* idx_B,
                                      tblis_b200_indexed_dpd_tensor* C, const label_type* idx_C,
                                tblis_b200_report* report);

/* Level-1 operations over indexed DPD tensors, the C entries of tblis::add /
 * dot / reduce / scale / set / shift over indexed_dpd_varray_view
 * (src/iface/1t/{add,dot,reduce,scale,set,shift}.cxx and src/internal/1t/indexed_dpd/). Entries act through
 * their factors as the reference's do: add scales B's entries by f*beta then
 * adds alpha*f_A*f_B*A_i to every B entry whose index values agree (a label
 * indexed in one tensor selects that slice of the other); dot sums
 * f_A*f_B*(A_i . B_j) over agreeing pairs; reduce combines the entries'
 * reductions scaled by their factors, idx counted from entry 0's data; scale
 * multiplies entry e by f_e*A.scalar, set writes f_e*alpha, shift writes
 * f_e*alpha + A.scalar*A (A.scalar*A only, when f_e == 0). Return 0 or an
 * error code. */
int tblis_b200_indexed_dpd_add(const tblis_b200_indexed_dpd_tensor* A, const label_type* idx_A,
                               tblis_b200_indexed_dpd_tensor* B, const label_type* idx_B);
int tblis_b200_indexed_dpd_dot(const tblis_b200_indexed_dpd_tensor* A, const label_type* idx_A,
                               const tblis_b200_indexed_dpd_tensor* B, const label_type* idx_B,
                               tblis_scalar* result);
int tblis_b200_indexed_dpd_reduce(reduce_t op, const tblis_b200_indexed_dpd_tensor* A, const label_type* idx_A,
                                  tblis_scalar* result, len_type* idx);
int tblis_b200_indexed_dpd_scale(tblis_b200_indexed_dpd_tensor* A, const label_type* idx_A);
int tblis_b200_indexed_dpd_set(const tblis_scalar* alpha, tblis_b200_indexed_dpd_tensor* A,
                               const label_type* idx_A);
int tblis_b200_indexed_dpd_shift(const tblis_scalar* alpha, tblis_b200_indexed_dpd_tensor* A,
                                 const label_type* idx_A);

/* Offset (from data), lengths and strides of one block (one irrep per
 * dimension), as dpd_varray_view::operator()(irreps) gives them
 * (dpd_marray_base.hpp:171-228). Returns 0 or an error code. */
/* A DPD contraction split across ranks (one process per GPU), with no
 * collective on the data path (no counterpart in the reference, which runs
 * on CPU threads). The unit of work is a row band of one irrep GEMM of
 * src/internal/3t/dpd/mult.cxx:308: the C blocks that share their AC (and
 * batch) irreps. Units go to ranks largest first onto the least loaded rank,
 * by FLOPs computed from the lengths alone, so every rank derives the same
 * split without a device.
 * tblis_b200_dpd_shard_plan (host-only): owner[t] = the rank that computes
 * the C block with irrep tuple t (t = sum_d irrep_d * nirrep^d, dimension 0
 * fastest; -1 where no block is stored; nirrep^ndim(C) entries), and, if
 * flops is not NULL, each rank's FLOPs (nranks entries).
 * tblis_b200_dpd_mult_shard: this rank's blocks of C = alpha*A*B + beta*C
 * (double tensors); the other blocks of C are left as they are. Both return
 * 0 or an error code. */
int tblis_b200_dpd_shard_plan(const tblis_b200_dpd_tensor* A, const label_type* idx_A,
                              const tblis_b200_dpd_tensor* B, const label_type* idx_B,
                              const tblis_b200_dpd_tensor* C, const label_type* idx_C,
                              int nranks, int* owner, double* flops);
int tblis_b200_dpd_mult_shard(const tblis_b200_dpd_tensor* A, const label_type* idx_A,
                              const tblis_b200_dpd_tensor* B, const label_type* idx_B,
                                    tblis_b200_dpd_tensor* C, const label_type* idx_C,
                              int nranks, int rank, tblis_b200_report* report);

int tblis_b200_dpd_block(const tblis_b200_dpd_tensor* A, const unsigned* irreps, len_type* len,
                         stride_type* stride, stride_type* offset);

/* Number of stored elements (all allowed blocks), or -1 on error. */
len_type tblis_b200_dpd_size(const tblis_b200_dpd_tensor* A);

/* ---- batches -------------------------------------------------------------- */

/* count independent contractions C[i] = alpha_i*A[i]*B[i] + beta_i*C[i] (each
 * as tblis_tensor_mult) in one grouped launch of the FP64 kernel; device data
 * only. The grouped plan (scatter vectors, tuned tile shape, CUDA graph) is
 * cached per set of shapes. Returns 0 or an error code. */
int tblis_b200_tensor_mult_batch(int count, const tblis_tensor* A, const label_type* const* idx_A,
                                 const tblis_tensor* B, const label_type* const* idx_B,
                                       tblis_tensor* C, const label_type* const* idx_C,
                                 tblis_b200_report* report);

/* ---- serving ---------------------------------------------------------------- */

/* A continuous-batching contraction server (no counterpart in the reference;
 * it serves the calls of src/iface/3t/mult.cxx:24-165 issued by a solver whose
 * operands stay device-resident). Requests queue in arrival order; a scheduler
 * thread admits them while their operand footprint (A, B and C extents) fits
 * the HBM budget, folds every admitted request into one grouped launch and
 * keeps up to `slots` launches in flight on separate streams, so requests that
 * arrive while others run start as soon as a slot and budget free up. Large
 * requests whose tolerance is at least 1e-13 run on the Ozaki INT8 path with
 * the slice count chosen from that tolerance; the rest run in FP64. A
 * request's result is the same alone and in any mix (every output tile is
 * computed by one CTA with a fixed k order). Tensors must be in device memory
 * and stay valid until the request completes; the tensor descriptors are
 * copied at submit. */
typedef struct tblis_b200_server tblis_b200_server;

typedef struct tblis_b200_server_stats
{
    int64_t completed;
    int64_t failed;
    int64_t batches;                 /* grouped launches */
    int64_t queued;                  /* waiting for admission */
    double mean_batch;               /* requests per launch */
    int max_concurrent_batches;      /* most launches seen in flight at once */
    double p50_ms, p99_ms, max_ms;   /* submit-to-completion latency */
    int64_t ozaki;                   /* requests run on the INT8 Ozaki path */
    int64_t shape_hits, shape_misses; /* requests whose shape (GEMM view and device
                                        scatter vectors) was cached / built */
} tblis_b200_server_stats;

tblis_b200_server* tblis_b200_server_create(size_t hbm_budget_bytes, int slots);
/* waits for every queued and running request, then frees the server */
void tblis_b200_server_destroy(tblis_b200_server* srv);
/* returns the request id (> 0), or -1 (last error: 7 = larger than the budget) */
int64_t tblis_b200_server_submit(tblis_b200_server* srv,
                                 const tblis_tensor* A, const label_type* idx_A,
                                 const tblis_tensor* B, const label_type* idx_B,
                                 const tblis_tensor* C, const label_type* idx_C, double tolerance);
/* 0 = done (the id is released), 1 = pending, else the request's error code */
int tblis_b200_server_poll(tblis_b200_server* srv, int64_t id, double* latency_ms);
int tblis_b200_server_wait(tblis_b200_server* srv, int64_t id, double* latency_ms);
int tblis_b200_server_get_stats(tblis_b200_server* srv, tblis_b200_server_stats* out);

/* Multi-GPU sharding (no counterpart in TBLIS, whose parallelism is TCI
 * threads on one node): a contraction split across `nranks` processes, one per
 * GPU, with no collective on the data path. C is partitioned along its longest
 * label that appears in exactly one of A and B; rank `rank` owns the range
 * [len*rank/nranks, len*(rank+1)/nranks) of that label and contracts the
 * matching slice of A (or B) into its slab of C. The slabs are disjoint and
 * cover C. Without such a label rank 0 computes everything.
 *
 * tblis_b200_shard_plan: host-only (needs no device): the cut label (0 when
 * none) and this rank's [begin, end).
 * tblis_b200_tensor_mult_shard: C's slab = alpha*A*B + beta*C's slab for
 * this rank, through the same path as tblis_tensor_mult; the rest of C is
 * untouched. Both return 0 or an error code. */
int tblis_b200_shard_plan(const tblis_tensor* A, const label_type* idx_A,
                          const tblis_tensor* B, const label_type* idx_B,
                          const tblis_tensor* C, const label_type* idx_C,
                          int nranks, int rank, char* label, len_type* begin, len_type* end);
int tblis_b200_tensor_mult_shard(const tblis_config* cfg,
                                 const tblis_tensor* A, const label_type* idx_A,
                                 const tblis_tensor* B, const label_type* idx_B,
                                       tblis_tensor* C, const label_type* idx_C,
                                 int nranks, int rank, tblis_b200_report* report);

/* No counterpart in the reference. tblis_tensor_mult for callers that cannot
 * let a library allocate device memory (their device memory is owned by
 * another allocator, or they must avoid cudaMalloc/cudaFree because those can
 * synchronise the device): the same FP64 DMMA kernel, with its scatter vectors
 * and split-K partial tiles in one fixed file-scope device array of
 * TBLIS_B200_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds
 * until exit. Where tblis_tensor_mult would run the FP64 path, it gives the
 * same result, with these differences: only double tensors (TB_ERR_TYPE = 2
 * otherwise), device memory only (host data is TB_ERR_ARG = 1: staging it
 * would allocate), no Ozaki or other method from a config. alpha == 0 or an
 * empty contracted extent sets or scales C by beta, as tblis_tensor_mult does.
 * A contraction whose scatter vectors exceed the array is rejected
 * (TB_ERR_SIZE = 5), and split-K is reduced until its partials fit. Calls
 * share the array: calls that overlap on the GPU race and must be
 * serialised. The first call on a device looks up the array's address; make
 * it before any stream capture. A failed call leaves C and its scalar as they
 * were. Returns 0 or an error code (also recorded as the last error). */
#define TBLIS_B200_NOALLOC_SCRATCH_BYTES ((size_t)32 << 20)
int tblis_b200_tensor_mult_noalloc(const tblis_tensor* A, const label_type* idx_A,
                                   const tblis_tensor* B, const label_type* idx_B,
                                         tblis_tensor* C, const label_type* idx_C);
size_t tblis_b200_noalloc_scratch_bytes(void);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif
