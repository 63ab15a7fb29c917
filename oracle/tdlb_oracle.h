/*
 * tdlb_oracle.h -- CPU restatement of tdLBCpp's lattice Boltzmann time step.
 *
 * TEST INFRASTRUCTURE ONLY (the parity oracle). Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, and only
 * as the checker. The product (tdlbcpp_b200/) never links or calls it.
 *
 * It restates, in plain C, the reference CPU ComputeUnit
 * (ComputeUnit<T,18,MemoryLayoutIJKL,EgglesSomers,{Simple|Esotwist},CPU>) with
 * the reference's data model: a ghosted AoS lattice whose Q holds moments
 * between steps, F (3 per cell), Nu and the O flag. Every operation keeps the
 * reference's arithmetic types (float variables, double literals promoting
 * the expression to double) and its term order, so that in FP32 it rounds
 * exactly as the reference compiled with -ffp-contract=off. It is pinned
 * against the reference compiled in place (oracle/_ref) and the reference's
 * golden streaming vectors by tests/test_oracle_pin.py.
 *
 * The API mirrors oracle/ref_shim/ref_capi.cpp (prefix tdlbo_ instead of
 * tdlbref_) so the two are interchangeable in tests.
 */
#ifndef TDLB_ORACLE_H
#define TDLB_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tdlbo_flow {
    double initialRho, nu, cs0, g3, alpha, beta;
    int32_t useLES;
    int32_t pad;
} tdlbo_flow;

/* Same layout as tdlb_marker in include/tdlb_b200.h. */
typedef struct tdlbo_marker {
    int64_t i, j, k;
    float iCartFraction, kCartFraction, uDelta, vDelta, wDelta, pad;
} tdlbo_marker;

void* tdlbo_create(int precision, int streaming, long x, long y, long z, const tdlbo_flow* flow, const char* unused);
void tdlbo_destroy(void* h);
long tdlbo_size(void* h);
int tdlbo_even_step(void* h);
void tdlbo_set_even_step(void* h, int even);
void tdlbo_set_nu(void* h, double nu);
void tdlbo_set_threads(int n);

void tdlbo_initialise(void* h, double rho);
void tdlbo_collision(void* h);
void tdlbo_bounce_back(void* h);
void tdlbo_streaming_push(void* h);
void tdlbo_moments(void* h);
void tdlbo_forcing(void* h, const tdlbo_marker* m, long n, double alpha, double beta);
void tdlbo_step(void* h, const tdlbo_marker* m, long n, double alpha, double beta);

void tdlbo_get_q(void* h, double* out);
void tdlbo_set_q(void* h, const double* in);
void tdlbo_get_f(void* h, double* out);
void tdlbo_set_f(void* h, const double* in);
void tdlbo_get_nu(void* h, double* out);
void tdlbo_set_nu_field(void* h, const double* in);
void tdlbo_get_o(void* h, uint8_t* out);
void tdlbo_get_moments(void* h, double* out);
void tdlbo_get_moments_range(void* h, long i0, long i1, double* out);
void tdlbo_transport(void* h);
void tdlbo_get_forcing_sums(void* h, double* out, long n);

/* Integer-coded transport known-answer tests, same contract as the
 * tdlbref_kat_* entry points of oracle/_ref. Values are exact in uint64. */
int tdlbo_kat_simple_stream(int push, long x, long y, long z, uint64_t* out);
int tdlbo_kat_esotwist(long x, long y, long z, int start_even, int nsteps, int moments_map, uint64_t* out);
int tdlbo_kat_esotwist_read(long x, long y, long z, int even, uint64_t* out);

#ifdef __cplusplus
}
#endif
#endif
