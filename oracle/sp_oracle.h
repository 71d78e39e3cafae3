/*
 * sp_oracle.h — CPU restatement (plain C, sequential) of SW2D's native single-porosity
 * explicit step, used ONLY as the checker of the CUDA path (tests, smoke check, the CPU
 * baseline leg of bench.py).  It is never linked into the product.
 *
 * It takes the same inputs as the product's C ABI (include/sw2d_b200.h) and keeps the
 * reference's data order: every loop runs over boundary edges, then internal edges, by
 * increasing index, exactly like src/sw2dSolver/models/sp/swSpHyp.cpp.  The restatement is
 * pinned against the reference compiled from its own sources (oracle/_ref, see Makefile).
 */
#ifndef SP_ORACLE_H
#define SP_ORACLE_H

#include "../include/sw2d_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sp_oracle sp_oracle;

sp_oracle* spo_create(const sw2d_mesh* mesh, const sw2d_params* params, const sw2d_cell_fields* fields,
                      const sw2d_bc_table* bc, const double* h0, const double* q0, const double* r0);
/* Runs up to n steps; returns the number taken, or a negative SW2D_E_* status. */
int spo_step(sp_oracle* o, int n);
void spo_get_state(const sp_oracle* o, double* h, double* q, double* r);
void spo_set_state(sp_oracle* o, const double* h, const double* q, const double* r);
double spo_time(const sp_oracle* o);
double spo_dt(const sp_oracle* o);
void spo_set_time(sp_oracle* o, double t, double dt);
/* Same names as sw2d_get_array; returns the element count, or -1 for an unknown name. */
long spo_get_array(const sp_oracle* o, const char* name, double* out);
/* 0: exp/log of the host libm (default, as the reference); 1: the portable exp/log of the
 * CUDA build (inria-internship-project-sw2d-enzyme_b200/csrc/portable_math.h). */
void spo_set_portable_math(sp_oracle* o, int on);
void spo_destroy(sp_oracle* o);

#ifdef __cplusplus
}
#endif

#endif
