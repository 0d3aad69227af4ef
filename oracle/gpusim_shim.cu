// ORACLE / BASELINE INFRASTRUCTURE ONLY: a thin C ABI over the reference's
// own plain complex128 GPU simulator (src/gpusim, compiled from the reference
// sources by oracle/Makefile into _ref/libgpusim_ref.so).  Used by tests/ to
// cross-check this package's uncompressed per-gate and fused paths, and by
// bench.py to time the reference's per-gate GPU path on the benchmark's gate
// list -- never by the product.
//
// gsref_apply dispatches one gate the way the reference does on a
// QuantumStateGpu: the named CNOT / SWAP / CZ gates call their kernels
// (src/cppsim/gate_named_two.hpp: _update_func_gpu), every other gate goes
// through QuantumGateMatrix::update_quantum_state's GPU branch
// (src/cppsim/gate_matrix.cpp:128-240): one target without controls ->
// single_qubit_dense_matrix_gate_host, one target with one control ->
// single_qubit_control_single_qubit_dense_matrix_gate_host, more controls ->
// multi_qubit_control_multi_qubit_dense_matrix_gate_host, several targets
// without controls -> multi_qubit_dense_matrix_gate_host.
#include <complex>
#include <cstdint>
#include <cstring>

#include <cuda_runtime.h>

#include "memory_ops.h"
#include "update_ops_cuda.h"

namespace {
void *g_stream = nullptr;  // the reference's stream object (allocate_cuda_stream_host)
}

extern "C" {

int gsref_init(unsigned int device) {
    if (!g_stream) g_stream = allocate_cuda_stream_host(1, device);
    return g_stream ? 0 : 1;
}

void *gsref_alloc(uint64_t dim) { return allocate_quantum_state_host((ITYPE)dim, 0); }

void gsref_free(void *state) { release_quantum_state_host(state, 0); }

void gsref_init_zero(void *state, uint64_t dim) { initialize_quantum_state_host(state, (ITYPE)dim, g_stream, 0); }

// matrix: row-major 2^ntargets x 2^ntargets, interleaved re, im
int gsref_apply(void *state, uint64_t dim, const char *name, uint32_t ntargets, const uint32_t *targets,
                uint32_t ncontrols, const uint32_t *controls, const uint32_t *cvals, const double *matrix) {
    const ITYPE d = (ITYPE)dim;
    if (!std::strcmp(name, "CNOT") && ntargets == 1 && ncontrols == 1) {
        CNOT_gate_host(controls[0], targets[0], state, d, g_stream, 0);
        return 0;
    }
    if (!std::strcmp(name, "CZ") && ntargets == 1 && ncontrols == 1) {
        CZ_gate_host(controls[0], targets[0], state, d, g_stream, 0);
        return 0;
    }
    if (!std::strcmp(name, "SWAP") && ntargets == 2 && ncontrols == 0) {
        SWAP_gate_host(targets[0], targets[1], state, d, g_stream, 0);
        return 0;
    }
    const CPPCTYPE *m = reinterpret_cast<const CPPCTYPE *>(matrix);
    UINT t[8], c[8], v[8];
    if (ntargets > 8 || ncontrols > 8) return 2;
    for (uint32_t i = 0; i < ntargets; ++i) t[i] = targets[i];
    for (uint32_t i = 0; i < ncontrols; ++i) {
        c[i] = controls[i];
        v[i] = cvals[i];
    }
    if (ntargets == 1) {
        if (ncontrols == 0) single_qubit_dense_matrix_gate_host(t[0], m, state, d, g_stream, 0);
        else if (ncontrols == 1)
            single_qubit_control_single_qubit_dense_matrix_gate_host(c[0], v[0], t[0], m, state, d, g_stream, 0);
        else
            multi_qubit_control_multi_qubit_dense_matrix_gate_host(c, v, ncontrols, t, ntargets, m, state, d,
                                                                   g_stream, 0);
        return 0;
    }
    if (ncontrols == 0) multi_qubit_dense_matrix_gate_host(t, ntargets, m, state, d, g_stream, 0);
    else
        multi_qubit_control_multi_qubit_dense_matrix_gate_host(c, v, ncontrols, t, ntargets, m, state, d, g_stream,
                                                               0);
    return 0;
}

// amplitudes [first, first + count) into host memory (2 * count doubles)
int gsref_get(const void *state, uint64_t first, uint64_t count, double *out) {
    cudaDeviceSynchronize();
    const cudaError_t e = cudaMemcpy(out, static_cast<const double *>(state) + 2 * first, count * 16,
                                     cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? 0 : 1;
}

int gsref_sync() { return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1; }

}  // extern "C"
