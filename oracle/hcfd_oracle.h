/* TEST INFRASTRUCTURE — the CPU oracle.  Only tests/, smoke() and bench.py's CPU legs may
 * load it, and only as the checker or the timed CPU baseline; the product never calls it.
 *
 * A plain-C restatement of the reference solver's Base layout
 * (Hasti-Jalal-Aldeen/CFD_Optimisations, src/Base/*.cpp), face loop by face loop, with the
 * same expression trees so that, built with the same compiler flags, it reproduces the
 * reference bit for bit.  Parity is pinned by tests/test_oracle.py against the reference's
 * shipped sols/Base_0.hsln and sols/Base_1.hsln and against the reference compiled here.
 *
 * The features the reference does not have (global CFL dt, local time stepping, the
 * Venkatakrishnan limiter, the L2 density residual and the wall pressure coefficient) are
 * defined here; their parity with the GPU solver is pinned only by this restatement.
 *
 * Built with HCFD_ORACLE_FP32 the same source steps in float (geometry rounded once from
 * double, compensated per-cell residual sums): the CPU counterpart of the FP32 path.  The
 * interface below is the same in both builds (doubles in and out).
 */
#ifndef HCFD_ORACLE_H
#define HCFD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hcfd_oracle hcfd_oracle;

enum { HCFD_OR_BJ = 0, HCFD_OR_VENKAT = 1 };
enum { HCFD_OR_FIXED_DT = 0, HCFD_OR_GLOBAL_CFL = 1, HCFD_OR_LOCAL_CFL = 2 };
enum { HCFD_OR_U = 0, HCFD_OR_Q = 1, HCFD_OR_PHI = 2, HCFD_OR_R = 3, HCFD_OR_G = 4,
       HCFD_OR_DTLOC = 5, HCFD_OR_IV = 6 };

/* Mesh arrays as the reference's Mesh exposes them (includes/Mesh.hpp:4-22).  Copied. */
hcfd_oracle* hcfd_oracle_create(int Nn, int Nc, int Nf, int Ncol, int NBCcol,
                                const int* coltag, const int* coloff, const double* nodes,
                                const int* fn_con, const int* fc_con,
                                const int* cn_off, const int* cn_con, double gma);
void hcfd_oracle_free(hcfd_oracle* o);

/* Euler::gather_BCs (src/Base/Euler.cpp:42-60): type = bcmap[coltag[colour]], state
 * qbc[bc] (primitive rho,u,v,p).  Types: 0 SYMMETRY, 1 WALL, 2 SUPINLET, 3 SUBINLET,
 * 4 SUPOUTLET, 5 SUBOUTLET (includes/Base/BoundaryConditions.hpp:6-13). */
int hcfd_oracle_gather_bcs(hcfd_oracle* o, const int* bcmap, int nbcmap, const double* qbc);
/* Euler::initialise (src/Base/Euler.cpp:62-77). */
int hcfd_oracle_initialise(hcfd_oracle* o, const double* qic);
/* Limiter freezing: steps 1..after compute the limiter; later steps reuse step `after`'s
 * limiter values with fresh gradients (0 = never freeze). */
int hcfd_oracle_set_freeze(hcfd_oracle* o, long long after);
/* kind HCFD_OR_BJ (src/Base/Limiter.cpp:19-77) or HCFD_OR_VENKAT with constant K. */
int hcfd_oracle_set_limiter(hcfd_oracle* o, int kind, double K);
/* One step.  mode HCFD_OR_FIXED_DT uses dt_or_cfl as dt (the reference's only mode);
 * HCFD_OR_GLOBAL_CFL uses the minimum over real cells of the local dt at CFL dt_or_cfl;
 * HCFD_OR_LOCAL_CFL advances each cell with its own dt.  *dt_used gets the global dt (or
 * the minimum local dt), *res_l2 the L2 density residual of this step's R.  Either
 * pointer may be NULL. */
int hcfd_oracle_step(hcfd_oracle* o, int mode, double dt_or_cfl, double* dt_used, double* res_l2);
/* Runs the phases of one step separately: 0 gradient, 1 limiter, 2 BC grads + limiter,
 * 3 flux, 4 add residuals (fixed dt), 5 clear R, 6 BC cells. */
int hcfd_oracle_phase(hcfd_oracle* o, int which, double dt);
/* Copies a field out.  U/Q/PHI/R: 4 x Nc, variable-major.  G: 4 x 2 x Nc.  DTLOC: Nc (local
 * dt at CFL 1 for real cells, 0 for ghosts).  IV: Nc. */
int hcfd_oracle_get(hcfd_oracle* o, int which, double* out);
int hcfd_oracle_set_U(hcfd_oracle* o, const double* u);
/* Replaces the limiter values, 4 x Nc variable-major (in effect while the limiter is frozen). */
int hcfd_oracle_set_phi(hcfd_oracle* o, const double* phi);
/* Wall pressure coefficient on the faces of one colour, in face order:
 * Cp = (p_CL - p_inf) / (0.5 rho_inf |u_inf|^2).  Returns the number of faces written. */
int hcfd_oracle_wall_cp(hcfd_oracle* o, int colour, double rho_inf, double p_inf,
                        double speed_inf, double* out);
/* Geometry after Euler's zero_bc_iv: rf Nf*4, nf Nf*2, Af Nf, If Nf, xc Nc*2, iv Nc. */
int hcfd_oracle_domain(hcfd_oracle* o, double* rf, double* nf, double* Af, double* If,
                       double* xc, double* iv);
int hcfd_oracle_nreal(hcfd_oracle* o);

#ifdef __cplusplus
}
#endif
#endif
