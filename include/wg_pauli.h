/*
 * wg_pauli.h -- C-ABI of the B200 (sm_100a) packed-Pauli kernels.
 *
 * This is the boundary between the host layers (the C++ drop-in classes of
 * include/wolfgang/, the Python module, ctypes callers) and the CUDA kernels in
 * libwgpauli.so.  Everything here is plain C: pointers, sizes, status codes.
 * No exception crosses it, and no CUDA or torch type appears in it (streams are
 * passed as the opaque wg_stream_t, which is the same pointer as cudaStream_t;
 * NULL means the legacy default stream).
 *
 * Data layout (the reference's PauliSum storage, include/wolfgang/pauli_sum.hpp
 * :125-138 of sghowell/wolfgang 0.2.3):
 *   x[t*words + q/64] bit (q%64) = X part of qubit q of term t; z likewise;
 *   I=00 X=10 Z=01 Y=11; words = ceil(num_qubits/64) (0 for 0 qubits);
 *   coefficients are complex128 stored as interleaved (re, im) doubles.
 * Device pointers must live on `device`.  Every entry point enqueues on
 * `stream`; entry points that return host values synchronise that stream.
 *
 * Status: WG_OK (0) or an error code; wg_last_error() returns the thread's
 * last message.  The C++ layer maps WG_ERR_INVALID to std::invalid_argument
 * (Python ValueError) and the others to std::runtime_error.
 */
#ifndef WG_PAULI_H
#define WG_PAULI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WG_OK 0
#define WG_ERR_INVALID 1  /* bad argument (reference: std::invalid_argument) */
#define WG_ERR_OOM 2      /* device memory exhausted */
#define WG_ERR_CUDA 3     /* CUDA runtime failure */
#define WG_ERR_TIMEOUT 4  /* a bounded device wait expired; the context stays usable */
#define WG_ERR_NO_DEVICE 5

#define WG_DTYPE_C128 0
#define WG_DTYPE_C64 1

typedef struct CUstream_st* wg_stream_t;

/* ------------------------------------------------------------ runtime ---- */
const char* wg_last_error(void);
int wg_abi_version(void);
/* Device discovery; replaces DevicePauliSum::cuda_status()
 * (include/wolfgang/device_pauli_sum.hpp:111, src/cuda/device_pauli_sum.cu:286-335). */
int wg_device_count(int* count);
int wg_runtime_versions(int* runtime_version, int* driver_version);
int wg_device_info(int ordinal, char* name, size_t name_cap, int* cc_major,
                   int* cc_minor, size_t* total_mem, int* sm_count);

/* ---------------------------------------------------------- autotuner ---- */
/* Tile shapes and schedules per shape class (new; no reference counterpart).
 * Tuned: the commutation kernel and its tile and rows per CTA (algo 0 of
 * wg_commutation_bits, 1-4 mask words), the bucketed sort's fine-bucket
 * target (wg_pauli_products / wg_simplify when wg_set_bucket_fine_target is
 * 0), and the group_commuting chunk length.  A class is (operation, mask
 * words, ceil log2 of the sizes).  Every candidate gives identical results.
 *   WG_TUNE_OFF     the measured defaults always;
 *   WG_TUNE_CACHED  (default) cached choices, the defaults elsewhere: no call
 *                   measures anything;
 *   WG_TUNE_SEARCH  the first call of a class with no cached choice times
 *                   every candidate on its own inputs (CUDA events, best of
 *                   two runs; it synchronises, so make that call outside
 *                   stream capture) and caches the fastest.
 * The cache is process-wide; export/import move it between processes as
 * text lines "<op> <words> <a> <b> <choice>" (op: commute, bucket, group_qwc,
 * group_full). */
#define WG_TUNE_OFF 0
#define WG_TUNE_CACHED 1
#define WG_TUNE_SEARCH 2
int wg_autotune_set_mode(int mode);
int wg_autotune_get_mode(int* mode);
/* Writes the cache as text (NUL-terminated) when buf has room;
 * *needed = bytes required including the NUL.  buf may be NULL. */
int wg_autotune_export(char* buf, size_t cap, size_t* needed);
/* Adds the classes of `text` to the cache (existing classes are replaced). */
int wg_autotune_import(const char* text);
int wg_autotune_clear(void);

/* ------------------------------------------------------------- memory ---- */
/* Stream-ordered allocations from the device's memory pool; replace the
 * per-call cudaMalloc/cudaFree of src/cuda/device_pauli_sum.cuh:70-113. */
int wg_malloc(int device, size_t bytes, wg_stream_t stream, void** out);
int wg_free(int device, void* ptr, wg_stream_t stream);
int wg_memcpy_htod(int device, void* dst, const void* src, size_t bytes, wg_stream_t stream);
int wg_memcpy_dtoh(int device, void* dst, const void* src, size_t bytes, wg_stream_t stream);
int wg_memcpy_dtod(int device, void* dst, const void* src, size_t bytes, wg_stream_t stream);
/* Device-to-host copy delivered in chunks: the buffer goes through pinned
 * staging and each chunk is handed, in order, to fn(user, chunk, chunk_bytes)
 * on the calling thread once it has landed (chunks are 8 MiB, the last one
 * shorter; a ring of three pinned buffers per call keeps two chunks in flight
 * while the caller consumes one).  Lets a caller build its own host container from the data without
 * first filling it (e.g. appending to a reserved std::vector).  Calls from
 * different threads run concurrently, each with its own staging and stream.
 * Ordering: the copies run on an internal stream that first waits for all
 * work enqueued on `stream` before the call (pass the stream whose kernels
 * write src; NULL = the legacy default stream).  Work enqueued on other
 * streams is not waited for.  Returns once every chunk has been handed over.
 * No reference counterpart (the reference downloads into resized vectors). */
typedef void (*wg_chunk_fn)(void* user, const void* chunk, size_t chunk_bytes);
int wg_memcpy_dtoh_chunked(int device, const void* src, size_t bytes, wg_chunk_fn fn, void* user,
                           wg_stream_t stream);
int wg_memset(int device, void* dst, int value, size_t bytes, wg_stream_t stream);
int wg_stream_synchronize(int device, wg_stream_t stream);
int wg_device_synchronize(int device);
/* Pointer validation for caller-owned statevectors; replaces the checks of
 * src/cuda/expectation_cuda.cu:211-250: is_device = -1 when the runtime does
 * not recognise the pointer, 0 for host memory, 1 for device memory; then
 * *device is its ordinal and in_one_allocation says whether the byte range
 * [ptr, ptr+bytes) lies in one allocation. */
int wg_pointer_check(const void* ptr, size_t bytes, int* is_device, int* device,
                     int* in_one_allocation);
/* Host-side fault injection for tests: the n-th next pool allocation (counting
 * from 1) reports WG_ERR_OOM without touching the device; n <= 0 disables. */
int wg_inject_alloc_failure(long n);
/* Number of kernels this library has launched in the process (all devices). */
int wg_kernel_launches(unsigned long long* count);
/* Per-kernel timing with CUDA events recorded on each kernel's launch stream
 * (off by default).  The report is "name:launches:total_ms;..." for the
 * kernels since the last report; it synchronises on the recorded events. */
int wg_profile_enable(int on);
int wg_profile_report(char* buf, size_t cap);

/* -------------------------------------------------------- commutation ---- */
/* Bit-packed all-pairs commutation matrix.  Replaces commutation_kernel
 * (src/cuda/commutation_cuda.cu:123-151) behind DevicePauliSum::commutes_with*
 * (include/wolfgang/device_pauli_sum.hpp:126-147) and PauliSum::commutes_with
 * (include/wolfgang/pauli_sum.hpp:77-79).
 * bits[row*pitch_words + c/32] bit (c%32) = 1 iff lhs term `row` commutes with
 * rhs term c; pitch_words >= ceil(n_rhs/32); padding bits are written 0.
 * algo: 0 = the autotuner's choice for the shape class (kernel, tile, rows
 * per CTA; see wg_autotune_set_mode), else a rule on the sizes and the word
 * count -- no term data is read, so the choice costs no synchronisation;
 * 1 = popcount/LOP3 with warp-ballot packing; 2 = bit-plane XOR over the lhs
 * support (up to 256 qubits; above that the call uses 1).  All algos give
 * identical bits. */
int wg_commutation_bits(int device, size_t words, const uint64_t* lhs_x,
                        const uint64_t* lhs_z, size_t n_lhs, const uint64_t* rhs_x,
                        const uint64_t* rhs_z, size_t n_rhs, uint32_t* bits,
                        size_t pitch_words, int algo, wg_stream_t stream);
/* Dense uint8 flags (the reference's layout: out[row*n_rhs + c] in {0,1}). */
int wg_bits_to_u8(int device, const uint32_t* bits, size_t rows, size_t cols,
                  size_t pitch_words, uint8_t* out, wg_stream_t stream);
/* Popcount consumers over the bit matrix; replace the reductions of
 * src/cuda/device_commutation_matrix.cu:84-141.  Any output may be NULL;
 * row_counts[rows] / col_counts[cols] are device buffers, *total is host. */
int wg_bits_count(int device, const uint32_t* bits, size_t rows, size_t cols,
                  size_t pitch_words, uint64_t* row_counts, uint64_t* col_counts,
                  uint64_t* total, wg_stream_t stream);
/* Dense uint8 commutation flags without any device allocation.  This entry
 * point has no counterpart in the reference.  It is for callers that cannot
 * allocate device memory while they run it: a host framework that owns and
 * accounts for the whole device budget, or a latency-critical loop that must
 * not call cudaMalloc/cudaFree (they synchronise the device).  The caller
 * passes the inputs and out[n_lhs*n_rhs]; the bit-packed matrix in between is
 * kept in one static 32 MiB device array that every GPU loading this library
 * holds until the process exits.  Limit: n_lhs * ceil(n_rhs/32) * 4 bytes
 * <= 32 MiB (up to 2^28 entries), larger requests fail with WG_ERR_INVALID.
 * The first call on a device resolves the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls share the array, so calls that overlap on the GPU (different
 * streams or threads) race; serialise them. */
int wg_commutation_u8_noalloc(int device, size_t words, const uint64_t* lhs_x,
                              const uint64_t* lhs_z, size_t n_lhs, const uint64_t* rhs_x,
                              const uint64_t* rhs_z, size_t n_rhs, uint8_t* out,
                              wg_stream_t stream);
/* The same counts over a dense uint8 flag matrix (DeviceCommutationMatrix). */
int wg_u8_count(int device, const uint8_t* flags, size_t rows, size_t cols,
                uint64_t* row_counts, uint64_t* col_counts, uint64_t* total,
                wg_stream_t stream);

/* ----------------------------------------------------------- simplify ---- */
/* PauliSum::simplify semantics (include/wolfgang/pauli_sum.hpp:57,
 * src/simplify.cpp:147-430); replaces src/cuda/simplify_cuda.cu:382-791.
 * Duplicate keys are summed in input order, |sum| <= atol + rtol*max|c| is
 * dropped, survivors come out in canonical order (x0,z0,x1,z1,...).  The
 * output buffers are allocated by the library on `device` (release with
 * wg_free); they are NULL when *out_terms == 0.  Synchronises `stream`. */
int wg_simplify(int device, size_t words, size_t n_terms, const uint64_t* x,
                const uint64_t* z, const double* coeffs, double atol, double rtol,
                uint64_t** out_x, uint64_t** out_z, double** out_coeffs,
                size_t* out_terms, wg_stream_t stream);

/* All-pairs products lhs*rhs (rhs acts first), PauliSum::matmul semantics
 * (include/wolfgang/pauli_sum.hpp:70-73, src/multiply.cpp:73-402); replaces
 * matmul_product_kernel (src/cuda/matmul_cuda.cu:36-87) + simplify.
 * mode: WG_PRODUCTS_RAW       products in nested-loop order (lhs outer);
 *       WG_PRODUCTS_SIMPLIFY  then simplify(atol, rtol);
 *       WG_PRODUCTS_FUSED     then sum and cull at |c| > 1e-12 (the threshold
 *                             of the reference's fused hash path,
 *                             src/multiply.cpp:107-261).
 * Outputs are allocated by the library as for wg_simplify. */
#define WG_PRODUCTS_RAW 0
#define WG_PRODUCTS_SIMPLIFY 1
#define WG_PRODUCTS_FUSED 2
int wg_pauli_products(int device, size_t words, const uint64_t* lhs_x,
                      const uint64_t* lhs_z, const double* lhs_c, size_t n_lhs,
                      const uint64_t* rhs_x, const uint64_t* rhs_z,
                      const double* rhs_c, size_t n_rhs, int mode, double atol,
                      double rtol, uint64_t** out_x, uint64_t** out_z,
                      double** out_coeffs, size_t* out_terms, wg_stream_t stream);

/* Prepared batch of products (new; no reference counterpart -- the per-call
 * path it replaces is wg_pauli_products, i.e. matmul_product_kernel +
 * simplify of src/cuda/matmul_cuda.cu:91-147, once per pair): n_pairs
 * products lhs_p * rhs_p of uneven sizes, all with `words` mask words, each
 * with PauliSum::matmul(simplify) semantics -- mode WG_PRODUCTS_SIMPLIFY
 * (simplify(atol, rtol) per pair) or WG_PRODUCTS_FUSED (cull at 1e-12).
 * Create reads the operands' masks once: it sorts every pair's products by
 * key, groups equal keys in nested-loop order and sizes all scratch and the
 * outputs (one slot per distinct key of a pair); it synchronises the device.
 * wg_products_batch_run then only enqueues kernels on `stream` -- no
 * allocation, host copy or host synchronisation -- so a run can be captured
 * in a CUDA graph and replayed.  Each run reads the coefficients through the
 * lhs_c/rhs_c device pointers given at create (their values may change
 * between runs; the masks must not) and writes pair p's simplified product,
 * in canonical order, to the batch's output slots (wg_products_batch_result)
 * and its term count to the device array of wg_products_batch_counts.  At
 * most 2^30 products per pair and fewer than 2^32 in all; coefficient buffers
 * 16-byte aligned (as every complex128 array is); runs of one batch must not
 * overlap. */
typedef struct wg_products_batch_s* wg_products_batch_t;
int wg_products_batch_create(int device, size_t words, size_t n_pairs, const uint64_t* const* lhs_x,
                             const uint64_t* const* lhs_z, const double* const* lhs_c, const size_t* n_lhs,
                             const uint64_t* const* rhs_x, const uint64_t* const* rhs_z,
                             const double* const* rhs_c, const size_t* n_rhs, int mode, double atol, double rtol,
                             wg_products_batch_t* batch, wg_stream_t stream);
int wg_products_batch_run(wg_products_batch_t batch, wg_stream_t stream);
/* Device pointers of pair p's output slots (valid until destroy; contents as
 * of the last run; x/z hold capacity*words words, coeffs 2*capacity doubles;
 * the first counts[p] terms are the result). */
int wg_products_batch_result(wg_products_batch_t batch, size_t pair, uint64_t** x, uint64_t** z,
                             double** coeffs, size_t* capacity);
/* Device array of n_pairs uint64 term counts, written by every run. */
int wg_products_batch_counts(wg_products_batch_t batch, uint64_t** counts);
/* Products and distinct (pair, key) slots of the batch. */
int wg_products_batch_info(wg_products_batch_t batch, size_t* n_products, size_t* n_keys);
/* Waits for the device, then frees the batch. */
int wg_products_batch_destroy(wg_products_batch_t batch);

/* Sort-reduce algorithm behind wg_simplify and the simplifying modes of
 * wg_pauli_products.  No reference counterpart (the reference has one sort);
 * both algorithms give identical results, bit for bit.
 *   WG_SORT_AUTO    (default) bucketed for 1-2 mask words, >= 2^20 items and
 *                   keys that vary in more than 8 (one word) or 5 (two words)
 *                   of their 8-bit digits; LSD otherwise;
 *   WG_SORT_LSD     multi-word LSD radix sort of full keys;
 *   WG_SORT_BUCKET  bucketed sort on 64-bit key codes (1-2 mask words, at most
 *                   255 significant key bits); falls back to WG_SORT_LSD when a
 *                   bucket of mixed keys stays over its capacity after being
 *                   split again, or one tie of key codes spans more than 16
 *                   distinct keys.
 * The setting is process-wide.  wg_last_sort_algorithm returns the algorithm
 * that produced the calling thread's last result (0 before any). */
#define WG_SORT_AUTO 0
#define WG_SORT_LSD 1
#define WG_SORT_BUCKET 2
int wg_set_sort_algorithm(int algo);
int wg_last_sort_algorithm(void);

/* Target items per fine bucket of WG_SORT_BUCKET (process-wide; 0 restores
 * the default, 896).  No reference counterpart; a tuning setting that changes
 * no result bit.  Fine buckets that come out over their capacity of 2048 items
 * are split again from their own samples before the final sort; a larger
 * target means fewer, fuller buckets.  Accepts 0 or 32..2048. */
int wg_set_bucket_fine_target(unsigned items);

/* Layout of WG_SORT_BUCKET's fine partition (process-wide).  1 (the default):
 * every fine bucket owns room for 2048 records and the partition pass writes
 * each item as it counts it, where that room (20 bytes a record) takes at
 * most a quarter of the device's memory; a coarse bucket with a fine bucket
 * over 2048 items is packed in a second pass.  0: always count first, then
 * pack (less memory).  Both give identical results.  No reference
 * counterpart; a tuning setting.  Accepts 0 or 1. */
int wg_set_bucket_one_pass(int on);

/* -------------------------------------------------------- expectation ---- */
/* <psi|H|psi> (PauliSum::expectation_statevector_complex{128,64},
 * include/wolfgang/pauli_sum.hpp:91-94; DevicePauliSum::expectation_statevector_*
 * include/wolfgang/device_pauli_sum.hpp:117-125); replaces
 * expectation_statevector_terms_kernel (src/cuda/expectation_cuda.cu:79-126).
 * Terms are grouped by x-mask so one streaming pass over psi serves every term
 * of a group.  An expectation plan holds the grouping for one operator
 * (device copies of its terms); it can be reused for many statevectors.
 * psi is a device buffer of 2^n_qubits complex128 or complex64 (FP64
 * accumulation either way).  n_qubits <= 63. */
typedef struct wg_expect_plan_s* wg_expect_plan_t;
int wg_expect_plan_create(int device, size_t n_qubits, size_t n_terms,
                          const uint64_t* x, const uint64_t* z, const double* coeffs,
                          wg_expect_plan_t* plan, wg_stream_t stream);
int wg_expect_plan_destroy(wg_expect_plan_t plan);
/* Replaces the coefficients of a plan (same terms, new values; device buffer
 * of 2*n_terms doubles in the plan's original term order). */
int wg_expect_plan_set_coeffs(wg_expect_plan_t plan, const double* coeffs, wg_stream_t stream);
int wg_expect_plan_info(wg_expect_plan_t plan, size_t* n_groups, size_t* n_terms);
/* Forward and adjoint in one x-grouped pass.  Any output may be NULL:
 *   result[2]        E = sum_k c_k <psi|P_k|psi> (device, complex128);
 *   term_values[T]   e_k = <psi|P_k|psi> (device, real FP64, original order) = dE/dc_k;
 *   hpsi[2^n]        H|psi> (device, complex128) = dE/dpsi* for Hermitian H. */
int wg_expect_plan_run(wg_expect_plan_t plan, const void* psi, int psi_dtype,
                       double* result, double* term_values, double* hpsi,
                       wg_stream_t stream);
/* One-shot drop-in: builds a plan, runs it, returns E on the host. */
int wg_expectation(int device, size_t n_qubits, size_t n_terms, const uint64_t* x,
                   const uint64_t* z, const double* coeffs, const void* psi,
                   int psi_dtype, double* result_host, wg_stream_t stream);

/* Batched uneven (H, psi) pairs in one persistent launch with a device work
 * queue (new; no reference counterpart).  Pair p uses plans[p] and psis[p]
 * (dtype psi_dtype for all pairs); outputs per pair as in wg_expect_plan_run
 * (arrays of device pointers; an array may be NULL, an element may be NULL).
 * The plan array and pointer arrays are host arrays. */
int wg_expect_batched(int device, size_t n_pairs, const wg_expect_plan_t* plans,
                      const void* const* psis, int psi_dtype, double* const* results,
                      double* const* term_values, double* const* hpsis,
                      wg_stream_t stream);

/* Prepared batch (new; no reference counterpart): the work tables for fixed
 * (plan, psi, outputs) pairs are uploaded once; wg_expect_batch_run then only
 * enqueues kernels on `stream` (no host synchronisation or host copies), so a
 * run can be captured in a CUDA graph and replayed.  Plans and buffers must
 * outlive the batch; runs of batches sharing a plan must not overlap. */
typedef struct wg_expect_batch_s* wg_expect_batch_t;
int wg_expect_batch_create(int device, size_t n_pairs, const wg_expect_plan_t* plans,
                           const void* const* psis, int psi_dtype, double* const* results,
                           double* const* term_values, double* const* hpsis,
                           wg_expect_batch_t* batch, wg_stream_t stream);
int wg_expect_batch_run(wg_expect_batch_t batch, wg_stream_t stream);
int wg_expect_batch_destroy(wg_expect_batch_t batch);

/* <H> over computational-basis counts (PauliSum::expectation_z_counts,
 * src/expectation.cpp:219-247): packed[rows*words] bitstrings (device),
 * counts[rows] (device).  Diagonal terms only.  Result on the host. */
int wg_expectation_z_counts(int device, size_t words, size_t n_terms,
                            const uint64_t* x, const uint64_t* z, const double* coeffs,
                            size_t rows, const uint64_t* packed, const double* counts,
                            double* result_host, wg_stream_t stream);

/* ------------------------------------------------------------ grouping ---- */
/* PauliSum::group_commuting(mode, "largest_first") (include/wolfgang/pauli_sum.hpp
 * :84-87, src/grouping.cpp:197-290): greedy first-fit over the deterministic
 * order (weight desc, canonical key, index).  mode_full = 0 for "qwc",
 * 1 for "full".  x/z are device buffers; order_out[n_terms] and
 * sizes_out[n_terms] are host buffers receiving term indices group after group
 * (placement order) and the group sizes. */
int wg_group_commuting(int device, size_t words, size_t n_terms, const uint64_t* x,
                       const uint64_t* z, int mode_full, size_t* order_out,
                       size_t* sizes_out, size_t* n_groups, wg_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* WG_PAULI_H */
