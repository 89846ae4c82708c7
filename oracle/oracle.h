/* Oracle tier B interface (test infrastructure only). */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrcInput {
    int N;
    const float *xrel;        /* N*3 cell-relative positions */
    const float *vel;         /* N*3 velocities (DPD), may be NULL */
    const int *cell;          /* N */
    const int *type;          /* N */
    int ncells;
    const double *cell_origin; /* ncells*3 */
    double dim[3];
    double cutoff;
    const int *tasks;         /* ntasks*4: type (1 self, 2 pair), sid, i, j */
    int ntasks;
    int ntypes;
    const float *radius;      /* ntypes */
    const int *pot_of_pair;   /* ntypes*ntypes, -1 none */
    const int *dpd_of_pair;   /* optional second (DPD) term per pair, or NULL */
    int npots;
    const int *pot_kind;      /* 0 table, 1 DPD */
    const unsigned *pot_flags;
    const int *pot_n;
    const float *pot_alpha;   /* npots*3 */
    const float *pot_abr;     /* npots*3: a, b, r0+1 */
    const int *pot_coef_off;  /* float offsets into coef */
    const float *coef;
    const float *dpd;         /* npots*4: alpha, gamma, sigma, 1/sqrt(dt) */
    const float *body;        /* ntypes*3 constant force, may be NULL */
    int cdim[3];              /* cells per axis */
    int pruning;              /* 0: reference pruning on non-cubic cells, 1: always, 2: never */
} OrcInput;

/* precision 32 or 64; f_out N*3; counts[3] = candidates, interacting, r<a skipped */
int orc_nonbond(int precision, const OrcInput *in, double *f_out, double *epot_out, long long *counts);
/* the same, plus the pair virial sum (x_first - x_second) (x) F_first, 9 doubles row-major */
int orc_nonbond_virial(int precision, const OrcInput *in, double *f_out, double *epot_out, long long *counts,
                       double *virial_out);

#ifdef __cplusplus
}
#endif
