// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// A C-ABI shim over the reference's own uncompressed FP64 CPU kernels (Qulacs
// "csim", src/csim/*.cpp of the reference tree), compiled from the reference
// sources where they lie by oracle/Makefile into oracle/_ref/libcsim_ref.so.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// it.  Nothing in the product links it.
//
// Every entry point forwards to exactly one reference function:
//   csimref_dense1      -> single_qubit_dense_matrix_gate        (src/csim/update_ops_matrix_dense_single.cpp)
//   csimref_dense2      -> double_qubit_dense_matrix_gate_c      (src/csim/update_ops_matrix_dense_double.cpp:42-62)
//   csimref_dense_multi -> multi_qubit_dense_matrix_gate         (src/csim/update_ops_matrix_dense_multi.cpp)
//   csimref_controlled  -> multi_qubit_control_multi_qubit_dense_matrix_gate
//                                                                (src/csim/update_ops_control_multi_target_multi.cpp)
//   csimref_cnot / cz / swap -> CNOT_gate / CZ_gate / SWAP_gate  (src/csim/update_ops_named_{CNOT,CZ,SWAP}.cpp)
//   csimref_norm_squared     -> state_norm_squared               (src/csim/stat_ops.cpp)
//   csimref_inner_product    -> state_inner_product              (src/csim/stat_ops.cpp)
//   csimref_init_zero        -> initialize_quantum_state         (src/csim/init_ops.cpp)
// State vectors are complex128 arrays (interleaved re, im) of length dim.
#include <complex>
#include <cstdint>

#include "csim/init_ops.hpp"
#include "csim/stat_ops.hpp"
#include "csim/update_ops.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

void csimref_dense1(unsigned t, const double* m, double* s, uint64_t dim) {
    single_qubit_dense_matrix_gate(t, reinterpret_cast<const CTYPE*>(m),
        reinterpret_cast<CTYPE*>(s), dim);
}

void csimref_dense2(
    unsigned t0, unsigned t1, const double* m, double* s, uint64_t dim) {
    double_qubit_dense_matrix_gate_c(t0, t1,
        reinterpret_cast<const CTYPE*>(m), reinterpret_cast<CTYPE*>(s), dim);
}

void csimref_dense_multi(const unsigned* targets, unsigned nt,
    const double* m, double* s, uint64_t dim) {
    multi_qubit_dense_matrix_gate(targets, nt,
        reinterpret_cast<const CTYPE*>(m), reinterpret_cast<CTYPE*>(s), dim);
}

void csimref_controlled(const unsigned* controls, const unsigned* cvals,
    unsigned nc, const unsigned* targets, unsigned nt, const double* m,
    double* s, uint64_t dim) {
    multi_qubit_control_multi_qubit_dense_matrix_gate(controls, cvals, nc,
        targets, nt, reinterpret_cast<const CTYPE*>(m),
        reinterpret_cast<CTYPE*>(s), dim);
}

void csimref_cnot(unsigned c, unsigned t, double* s, uint64_t dim) {
    CNOT_gate(c, t, reinterpret_cast<CTYPE*>(s), dim);
}

void csimref_cz(unsigned c, unsigned t, double* s, uint64_t dim) {
    CZ_gate(c, t, reinterpret_cast<CTYPE*>(s), dim);
}

void csimref_swap(unsigned a, unsigned b, double* s, uint64_t dim) {
    SWAP_gate(a, b, reinterpret_cast<CTYPE*>(s), dim);
}

double csimref_norm_squared(const double* s, uint64_t dim) {
    return state_norm_squared(reinterpret_cast<const CTYPE*>(s), dim);
}

void csimref_inner_product(
    const double* bra, const double* ket, uint64_t dim, double* out2) {
    CTYPE v = state_inner_product(reinterpret_cast<const CTYPE*>(bra),
        reinterpret_cast<const CTYPE*>(ket), dim);
    out2[0] = v.real();
    out2[1] = v.imag();
}

void csimref_init_zero(double* s, uint64_t dim) {
    initialize_quantum_state(reinterpret_cast<CTYPE*>(s), dim);
}

int csimref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
