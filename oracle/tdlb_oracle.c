/*
 * tdlb_oracle.c -- CPU restatement of tdLBCpp's lattice Boltzmann time step
 * (TEST INFRASTRUCTURE ONLY; see tdlb_oracle.h).
 *
 * Built by oracle/Makefile (`make -C oracle port`) with -ffp-contract=off.
 * Cell loops of collision/moments/streaming are OpenMP-parallel (each cell is
 * independent there); forcing() is sequential in marker order, as the
 * reference's is (Forcing.hpp:72-157).
 */
#include "tdlb_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Population slots, Header.h:70-100 (18 moving populations, no rest one). */
enum { Q01, Q02, Q03, Q04, Q05, Q06, Q07, Q08, Q09, Q10, Q11, Q12, Q13, Q14, Q15, Q16, Q17, Q18 };
/* Moment slots, Header.h:103-121. */
enum { M01, M02, M03, M04, M05, M06, M07, M08, M09, M10, M11, M12, M13, M14, M15, M16, M17, M18 };

/* Lattice vectors c_d in slot order (Header.h:70-100 comments). */
static const int C_DIR[18][3] = {
    {+1, 0, 0}, {-1, 0, 0}, {0, +1, 0}, {0, -1, 0}, {0, 0, +1}, {0, 0, -1},
    {+1, +1, 0}, {-1, -1, 0}, {+1, 0, +1}, {-1, 0, -1}, {0, +1, +1}, {0, -1, -1},
    {+1, -1, 0}, {-1, +1, 0}, {+1, 0, -1}, {-1, 0, +1}, {0, +1, -1}, {0, -1, +1},
};

#define R float
#define S(name) name##_f32
#include "tdlb_oracle_body.inc"
#undef R
#undef S
#define R double
#define S(name) name##_f64
#include "tdlb_oracle_body.inc"
#undef R
#undef S

typedef struct Handle {
    int precision;
    void* lat;
} Handle;

#define LAT32(h) ((Lattice_f32*)((Handle*)(h))->lat)
#define LAT64(h) ((Lattice_f64*)((Handle*)(h))->lat)
#define DISPATCH(h, expr32, expr64) do { if (((Handle*)(h))->precision == 4) { expr32; } else { expr64; } } while (0)

#define ALLOC_LATTICE(L, R_T, st, x_, y_, z_, fl)                                  \
    do {                                                                          \
        L = (R_T*)calloc(1, sizeof(*L));                                          \
        L->x = x_; L->y = y_; L->z = z_;                                          \
        L->xg = x_ + 2; L->yg = y_ + 2; L->zg = z_ + 2;                           \
        L->size = (size_t)L->xg * (size_t)L->yg * (size_t)L->zg;                  \
        L->streaming = st; L->evenStep = 1;                                       \
        const tdlbo_flow* fl_ = (fl);                                             \
        if (fl_) {                                                                \
            L->initialRho = fl_->initialRho; L->nu = fl_->nu; L->cs0 = fl_->cs0;  \
            L->g3 = fl_->g3; L->alpha = fl_->alpha; L->beta = fl_->beta;          \
            L->useLES = fl_->useLES ? 1 : 0;                                      \
        }                                                                         \
        L->Q = calloc(L->size * 18, sizeof(*L->Q));                               \
        L->Qtmp = calloc(L->size * 18, sizeof(*L->Q));                            \
        L->F = calloc(L->size * 3, sizeof(*L->F));                                \
        L->Nu = calloc(L->size, sizeof(*L->Nu));                                  \
        L->O = calloc(L->size, 1);                                                \
        L->Olast = calloc(L->size, 1);                                            \
    } while (0)

#define FREE_LATTICE(L) do { free(L->Q); free(L->Qtmp); free(L->F); free(L->Nu); free(L->O); free(L->Olast); free(L->sums); free(L); } while (0)

void tdlbo_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

void* tdlbo_create(int precision, int streaming, long x, long y, long z, const tdlbo_flow* flow, const char* unused) {
    (void)unused;
    if ((precision != 4 && precision != 8) || (streaming != 0 && streaming != 1)) return NULL;
    if (x < 1 || y < 1 || z < 1) return NULL;
    Handle* h = (Handle*)calloc(1, sizeof(Handle));
    h->precision = precision;
    if (precision == 4) { Lattice_f32* L; ALLOC_LATTICE(L, Lattice_f32, streaming, x, y, z, flow); h->lat = L; }
    else { Lattice_f64* L; ALLOC_LATTICE(L, Lattice_f64, streaming, x, y, z, flow); h->lat = L; }
    return h;
}

void tdlbo_destroy(void* h) {
    if (!h) return;
    DISPATCH(h, FREE_LATTICE(LAT32(h)), FREE_LATTICE(LAT64(h)));
    free(h);
}

static long tdlbo_size_x(void* h) { long s; DISPATCH(h, s = (long)LAT32(h)->x, s = (long)LAT64(h)->x); return s; }
long tdlbo_size(void* h) { long s; DISPATCH(h, s = (long)LAT32(h)->size, s = (long)LAT64(h)->size); return s; }
int tdlbo_even_step(void* h) { int e; DISPATCH(h, e = LAT32(h)->evenStep, e = LAT64(h)->evenStep); return e; }
void tdlbo_set_even_step(void* h, int even) { DISPATCH(h, LAT32(h)->evenStep = even != 0, LAT64(h)->evenStep = even != 0); }
void tdlbo_set_nu(void* h, double nu) { DISPATCH(h, LAT32(h)->nu = (float)nu, LAT64(h)->nu = nu); }

void tdlbo_initialise(void* h, double rho) { DISPATCH(h, initialise_f32(LAT32(h), (float)rho), initialise_f64(LAT64(h), rho)); }
void tdlbo_collision(void* h) { DISPATCH(h, collision_f32(LAT32(h)), collision_f64(LAT64(h))); }
/* Simple's ghost-face bounce-back (Boundary.hpp:18-250) only writes ghost
 * cells that no later stage reads; Esotwist's is empty (Boundary.hpp:14). */
void tdlbo_bounce_back(void* h) { (void)h; }
void tdlbo_streaming_push(void* h) { DISPATCH(h, streaming_push_f32(LAT32(h)), streaming_push_f64(LAT64(h))); }
void tdlbo_moments(void* h) { DISPATCH(h, moments_f32(LAT32(h)), moments_f64(LAT64(h))); }
void tdlbo_forcing(void* h, const tdlbo_marker* m, long n, double alpha, double beta) {
    DISPATCH(h, forcing_f32(LAT32(h), m, n, (float)alpha, (float)beta), forcing_f64(LAT64(h), m, n, alpha, beta));
}
void tdlbo_step(void* h, const tdlbo_marker* m, long n, double alpha, double beta) {
    tdlbo_collision(h);
    tdlbo_bounce_back(h);
    tdlbo_streaming_push(h);
    tdlbo_moments(h);
    tdlbo_forcing(h, m, n, alpha, beta);
}

#define COPY_OUT(L, arr, n, out) do { for (size_t c = 0; c < (n); c++) (out)[c] = (double)(L)->arr[c]; } while (0)
#define COPY_IN(L, arr, n, in, R_T) do { for (size_t c = 0; c < (n); c++) (L)->arr[c] = (R_T)(in)[c]; } while (0)

void tdlbo_get_q(void* h, double* out) { DISPATCH(h, COPY_OUT(LAT32(h), Q, LAT32(h)->size * 18, out), COPY_OUT(LAT64(h), Q, LAT64(h)->size * 18, out)); }
void tdlbo_set_q(void* h, const double* in) { DISPATCH(h, COPY_IN(LAT32(h), Q, LAT32(h)->size * 18, in, float), COPY_IN(LAT64(h), Q, LAT64(h)->size * 18, in, double)); }
void tdlbo_get_f(void* h, double* out) { DISPATCH(h, COPY_OUT(LAT32(h), F, LAT32(h)->size * 3, out), COPY_OUT(LAT64(h), F, LAT64(h)->size * 3, out)); }
void tdlbo_set_f(void* h, const double* in) { DISPATCH(h, COPY_IN(LAT32(h), F, LAT32(h)->size * 3, in, float), COPY_IN(LAT64(h), F, LAT64(h)->size * 3, in, double)); }
void tdlbo_get_nu(void* h, double* out) { DISPATCH(h, COPY_OUT(LAT32(h), Nu, LAT32(h)->size, out), COPY_OUT(LAT64(h), Nu, LAT64(h)->size, out)); }
void tdlbo_set_nu_field(void* h, const double* in) { DISPATCH(h, COPY_IN(LAT32(h), Nu, LAT32(h)->size, in, float), COPY_IN(LAT64(h), Nu, LAT64(h)->size, in, double)); }
/* The spread sums (sum of w*(j + F/2) minus rho_sum*u, 3 per marker) of the
 * last forcing() call, in marker order. */
void tdlbo_get_forcing_sums(void* h, double* out, long n) {
    DISPATCH(h, memcpy(out, LAT32(h)->sums, sizeof(double) * 3 * (size_t)n), memcpy(out, LAT64(h)->sums, sizeof(double) * 3 * (size_t)n));
}

void tdlbo_get_o(void* h, uint8_t* out) {
    DISPATCH(h, memcpy(out, LAT32(h)->Olast, LAT32(h)->size), memcpy(out, LAT64(h)->Olast, LAT64(h)->size));
}

/* Interior moments through the reference's read accessor (plain Q for
 * Simple, the esoteric read map for Esotwist), interior cells in (i, j, k)
 * order, 18 per cell. */
#define GET_MOMENTS(L, out, i_lo, i_hi)                                            \
    do {                                                                           \
        size_t c_ = 0;                                                             \
        for (long i = 1 + (i_lo); i <= (i_hi); i++)                                \
            for (long j = 1; j <= (L)->yg - 2; j++)                                \
                for (long k = 1; k <= (L)->zg - 2; k++, c_++) {                    \
                    __typeof__((L)->Q[0]) q_[18];                                  \
                    if ((L)->streaming == 0) {                                     \
                        size_t e_ = ((size_t)i * (L)->yg + j) * (L)->zg + k;       \
                        for (int l = 0; l < 18; l++) q_[l] = (L)->Q[e_ * 18 + l];  \
                    } else {                                                       \
                        GET_MOMENTS_ESO(L, i, j, k, q_);                           \
                    }                                                              \
                    for (int l = 0; l < 18; l++) (out)[c_ * 18 + l] = q_[l];       \
                }                                                                  \
    } while (0)

/* The same for the interior slab i0 <= i < i1 (0-based interior i), so that
 * a large lattice can be compared one slab at a time. */
void tdlbo_get_moments_range(void* h, long i0, long i1, double* out) {
    if (((Handle*)h)->precision == 4) {
        Lattice_f32* L = LAT32(h);
        if (i0 < 0) i0 = 0;
        if (i1 > L->xg - 2) i1 = L->xg - 2;
#define GET_MOMENTS_ESO(L, i, j, k, q) eso_read_f32(L, (L)->Q, i, j, k, (L)->evenStep, q)
        GET_MOMENTS(L, out, i0, i1);
#undef GET_MOMENTS_ESO
    } else {
        Lattice_f64* L = LAT64(h);
        if (i0 < 0) i0 = 0;
        if (i1 > L->xg - 2) i1 = L->xg - 2;
#define GET_MOMENTS_ESO(L, i, j, k, q) eso_read_f64(L, (L)->Q, i, j, k, (L)->evenStep, q)
        GET_MOMENTS(L, out, i0, i1);
#undef GET_MOMENTS_ESO
    }
}

void tdlbo_get_moments(void* h, double* out) { tdlbo_get_moments_range(h, 0, tdlbo_size_x(h), out); }

/* One transport-only step on the current Q: Simple push
 * (StreamingSimple.hpp:257-307) or, for Esotwist, AccessField read + write
 * for every interior cell followed by the parity flip (the step with an
 * identity collision). */
void tdlbo_transport(void* h) {
#define TRANSPORT(L, SFX)                                                                  \
    do {                                                                                   \
        if ((L)->streaming == 0) { stream_simple_##SFX(L, 1); break; }                     \
        for (long i = 1; i <= (L)->xg - 2; i++)                                            \
            for (long j = 1; j <= (L)->yg - 2; j++)                                        \
                for (long k = 1; k <= (L)->zg - 2; k++) {                                  \
                    __typeof__((L)->Q[0]) q_[18];                                          \
                    eso_read_##SFX(L, (L)->Q, i, j, k, (L)->evenStep, q_);                 \
                    eso_write_##SFX(L, (L)->Q, i, j, k, (L)->evenStep, q_);                \
                }                                                                          \
        (L)->evenStep = !(L)->evenStep;                                                    \
    } while (0)
    if (((Handle*)h)->precision == 4) { Lattice_f32* L = LAT32(h); TRANSPORT(L, f32); }
    else { Lattice_f64* L = LAT64(h); TRANSPORT(L, f64); }
#undef TRANSPORT
}

/* ---- integer-coded transport KATs (values exact in double) ---- */

static void fill_coded_f64(Lattice_f64* L) {
    /* tests/Params/ParamsCommon.hpp:168-206 coding, offset 0, two digits */
    for (long i = 0; i < L->xg; i++)
        for (long j = 0; j < L->yg; j++)
            for (long k = 0; k < L->zg; k++) {
                double base = (double)(((i * 100 + j) * 100 + k) * 100);
                size_t c = idx_f64(L, i, j, k);
                for (int l = 0; l < 18; l++) L->Q[c * 18 + l] = base + l;
            }
}

static void dump_u64(const Lattice_f64* L, uint64_t* out) {
    for (size_t c = 0; c < L->size * 18; c++) out[c] = (uint64_t)L->Q[c];
}

int tdlbo_kat_simple_stream(int push, long x, long y, long z, uint64_t* out) {
    if (x + 2 > 99 || y + 2 > 99 || z + 2 > 99) return 1;
    Lattice_f64* L;
    ALLOC_LATTICE(L, Lattice_f64, 0, x, y, z, (const tdlbo_flow*)NULL);
    fill_coded_f64(L);
    stream_simple_f64(L, push ? 1 : 0);
    dump_u64(L, out);
    FREE_LATTICE(L);
    return 0;
}

int tdlbo_kat_esotwist(long x, long y, long z, int start_even, int nsteps, int moments_map, uint64_t* out) {
    if (x + 2 > 99 || y + 2 > 99 || z + 2 > 99) return 1;
    Lattice_f64* L;
    ALLOC_LATTICE(L, Lattice_f64, 1, x, y, z, (const tdlbo_flow*)NULL);
    fill_coded_f64(L);
    L->evenStep = start_even != 0;
    for (int s = 0; s < nsteps; s++) {
        for (long i = 1; i <= L->xg - 2; i++)
            for (long j = 1; j <= L->yg - 2; j++)
                for (long k = 1; k <= L->zg - 2; k++) {
                    double q[18];
                    eso_read_f64(L, L->Q, i, j, k, L->evenStep, q);
                    if (moments_map) eso_write_moments_f64(L, L->Q, i, j, k, L->evenStep, q);
                    else eso_write_f64(L, L->Q, i, j, k, L->evenStep, q);
                }
        if (!moments_map) L->evenStep = !L->evenStep;
    }
    dump_u64(L, out);
    FREE_LATTICE(L);
    return 0;
}

int tdlbo_kat_esotwist_read(long x, long y, long z, int even, uint64_t* out) {
    if (x + 2 > 99 || y + 2 > 99 || z + 2 > 99) return 1;
    Lattice_f64* L;
    ALLOC_LATTICE(L, Lattice_f64, 1, x, y, z, (const tdlbo_flow*)NULL);
    fill_coded_f64(L);
    size_t c = 0;
    for (long i = 1; i <= L->xg - 2; i++)
        for (long j = 1; j <= L->yg - 2; j++)
            for (long k = 1; k <= L->zg - 2; k++, c++) {
                double q[18];
                eso_read_f64(L, L->Q, i, j, k, even != 0, q);
                for (int l = 0; l < 18; l++) out[c * 18 + l] = (uint64_t)q[l];
            }
    FREE_LATTICE(L);
    return 0;
}
