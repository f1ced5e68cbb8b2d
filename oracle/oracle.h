/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * Scalar CPU restatement of the packed-Pauli semantics of sghowell/wolfgang
 * 0.2.3.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference arm may load this library.  The product path (wolfgang_b200) never
 * links or calls it.
 *
 * Layout conventions (reference include/wolfgang/pauli_sum.hpp:125-138,
 * docs/architecture/semantic_contracts.md:7-32):
 *   x[t*words + q/64] bit (q%64) is the X part of qubit q of term t, z likewise;
 *   I=00, X=10, Z=01, Y=11; coefficients are interleaved (re, im) doubles.
 *
 * Every function returns 0 on success, 1 on invalid argument (message in
 * or_last_error()).
 */
#ifndef WOLFGANG_ORACLE_H
#define WOLFGANG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

const char* or_last_error(void);

/* std::abs(std::complex<double>) as the reference evaluates it (glibc hypot). */
double or_abs(double re, double im);

/* PauliSum::simplify (src/simplify.cpp:147-430).  Outputs must hold T terms. */
int or_simplify(size_t T, size_t words, const uint64_t* x, const uint64_t* z,
                const double* c, double atol, double rtol, uint64_t* ox,
                uint64_t* oz, double* oc, size_t* out_terms);

/* PauliSum::matmul (src/multiply.cpp:73-402).  Outputs must hold nl*nr terms.
 * simplify=0 emits products in nested-loop order. */
int or_matmul(size_t nl, size_t nr, size_t words, const uint64_t* lx,
              const uint64_t* lz, const double* lc, const uint64_t* rx,
              const uint64_t* rz, const double* rc, int simplify,
              uint64_t* ox, uint64_t* oz, double* oc, size_t* out_terms);

/* Products of matmul+simplify restricted to canonical keys k with
 * key_lo <= k < key_hi (keys given as 2*words words in canonical significance
 * order x0,z0,x1,z1,...).  Same summation order and cull as or_matmul, so the
 * result equals the matching slice of or_matmul's output.  Used to check the
 * full-size product workload one key range at a time.  cap = output capacity
 * (terms); a range with more survivors fails. */
int or_matmul_keyrange(size_t nl, size_t nr, size_t words, const uint64_t* lx,
                       const uint64_t* lz, const double* lc, const uint64_t* rx,
                       const uint64_t* rz, const double* rc,
                       const uint64_t* key_lo, const uint64_t* key_hi,
                       int fused_threshold, size_t cap, uint64_t* ox,
                       uint64_t* oz, double* oc, size_t* out_terms);

/* Whether PauliSum::matmul would take its fused hash path
 * (src/multiply.cpp:29-69, :107-109, :179-181). */
int or_matmul_uses_fused_path(size_t nl, size_t nr, size_t words,
                              const uint64_t* lx, const uint64_t* lz,
                              const uint64_t* rx, const uint64_t* rz,
                              int simplify);

/* PauliSum::commutes_with (src/commute.cpp:27-93,
 * src/detail/commutation.hpp:10-46).  out[l*nr + r] = 1 iff the pair commutes. */
int or_commutes(size_t nl, size_t nr, size_t words, const uint64_t* lx,
                const uint64_t* lz, const uint64_t* rx, const uint64_t* rz,
                uint8_t* out);

/* PauliSum::group_commuting (src/grouping.cpp:197-290).  mode_full = 0 for
 * "qwc", 1 for "full".  order_out[T] lists term indices group after group in
 * placement order; sizes_out[T] receives the group sizes. */
int or_group_commuting(size_t T, size_t words, const uint64_t* x,
                       const uint64_t* z, int mode_full, size_t* order_out,
                       size_t* sizes_out, size_t* n_groups);

/* PauliSum::expectation_statevector_complex{128,64}
 * (src/expectation.cpp:37-155, :209-217).  dtype 0 = complex128, 1 = complex64.
 * out[2] = (re, im).  Summation order is the reference's. */
int or_expectation(size_t T, size_t n_qubits, const uint64_t* x,
                   const uint64_t* z, const double* c, const void* psi,
                   int dtype, double* out);

/* Per-term <psi|P_k|psi> (real), the reference's per-term `term_expectation`
 * (src/expectation.cpp:116-153) with compensated (Neumaier) summation, used as
 * the high-accuracy FP64 reference for dE/dc_k. */
int or_term_expectations(size_t T, size_t n_qubits, const uint64_t* x,
                         const uint64_t* z, const void* psi, int dtype,
                         double* out);

/* H|psi>, with P|b> = i^{popc(x&z)} (-1)^{popc(z&b)} |b^x> (the convention of
 * src/expectation.cpp:121-150).  psi and out are complex128. */
int or_hpsi(size_t T, size_t n_qubits, const uint64_t* x, const uint64_t* z,
            const double* c, const double* psi, double* out);

/* (H|psi>)[idx[i]] for i < m: or_hpsi at the listed amplitudes only (for
 * statevectors whose full H|psi> the oracle cannot afford). */
int or_hpsi_at(size_t T, size_t n_qubits, const uint64_t* x, const uint64_t* z,
               const double* c, const double* psi, size_t m, const uint64_t* idx,
               double* out);

/* PauliSum::expectation_z_counts (src/expectation.cpp:219-247) with bitstrings
 * already packed (row-major, `words` words per row). */
int or_expectation_z_counts(size_t T, size_t words, const uint64_t* x,
                            const uint64_t* z, const double* c, size_t rows,
                            const uint64_t* packed, const double* counts,
                            double* out);

#ifdef __cplusplus
}
#endif
#endif
