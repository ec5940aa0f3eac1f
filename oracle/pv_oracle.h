/* pv_oracle.h — CPU restatement of the PointVortex hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the oracle the CUDA product is checked against. Only tests/,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py may load it.
 *
 * Parity is pinned two ways: against the unmodified reference compiled into oracle/_ref/
 * (tests/test_oracle.py) and against the golden vectors of the reference's own tests
 * (tests/tests.cpp, tests/audit_tests.cpp of jplaurie/PointVortex; tests/test_golden.py).
 *
 * Status codes: 0 ok, 1 invalid_argument, 2 out_of_range, 3 runtime_error, 4 logic_error.
 */
#ifndef PV_ORACLE_H
#define PV_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int geometry; /* 0 infinite, 1 periodic, 2 disk */
    double core_radius;
    double box_length_x;
    double box_length_y;
    int image_layers;
    double disk_radius;
    double absolute_tolerance;
    double relative_tolerance;
    double minimum_time_step;
    double maximum_time_step;
    int dipole_removal;
    double dipole_removal_distance;
    int dipole_reinjection;
    uint64_t random_seed;
} pvo_params;

typedef struct {
    size_t first;
    size_t second; /* == n for a disk wall-image candidate */
    double distance_squared;
} pvo_candidate;

const char *pvo_last_error(void);

int pvo_evaluate_range(const pvo_params *p, const double *x, const double *y, const double *g,
                       size_t n, size_t begin, size_t end, double *u, double *v);
int pvo_evaluate(const pvo_params *p, const double *x, const double *y, const double *g,
                 size_t n, double *u, double *v);
int pvo_hamiltonian(const pvo_params *p, const double *x, const double *y, const double *g,
                    size_t n, double *out);
int pvo_invariants(const pvo_params *p, const double *x, const double *y, const double *g,
                   size_t n, double *out5);

/* Integrator state: initial/temporary positions, 7 stage fields and the FSAL flag. */
typedef struct pvo_stepper pvo_stepper;
pvo_stepper *pvo_stepper_create(const pvo_params *p, size_t n);
void pvo_stepper_destroy(pvo_stepper *s);
void pvo_stepper_invalidate(pvo_stepper *s);
int pvo_rk4_step(pvo_stepper *s, double *x, double *y, const double *g, size_t n, double dt);
int pvo_dopri5_step(pvo_stepper *s, double *x, double *y, const double *g, size_t n, double dt,
                    double *out4);
/* Number of velocity evaluations the stepper has made (the reference's CountingKernel). */
size_t pvo_stepper_evaluations(const pvo_stepper *s);

/* Close-dipole candidate scan; writes at most cap candidates in scan order, returns the full
 * count in *count. */
int pvo_dipole_scan(const pvo_params *p, const double *x, const double *y, const double *g,
                    size_t n, pvo_candidate *out, size_t cap, size_t *count);

#ifdef __cplusplus
}
#endif
#endif
