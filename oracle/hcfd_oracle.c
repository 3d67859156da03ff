/* TEST INFRASTRUCTURE — the CPU oracle (see hcfd_oracle.h).  Never linked into the product.
 *
 * Restates the reference's Base layout (Hasti-Jalal-Aldeen/CFD_Optimisations) in C.  Each
 * function cites the reference lines it follows.  Arrays keep the reference's layouts:
 * state variable-major U[var][cell], gradients G[var][dim*Nc + cell], face geometry
 * face-major.  Expression trees are kept as written in the reference (operand order and
 * association), so the same compiler and flags give the same floating-point results.
 */
#include "hcfd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NV 4
#define ND 2

/* The arithmetic of the step (state, gradients, limiter values, fluxes, residuals).  The
 * default build is double and restates the reference.  The HCFD_ORACLE_FP32 build is the CPU
 * counterpart of the library's FP32 path: geometry computed in double and rounded once,
 * state and step arithmetic in IEEE float, each cell's residual summed with a compensated
 * two-sum in the reference's face order, dt minima and the residual norm in double.  (The
 * library's FP32 kernels use the hardware's approximate division and square root, so the two
 * agree to a few units in the last place per operation, not bit for bit.) */
#ifdef HCFD_ORACLE_FP32
typedef float real;
#define RSQRT sqrtf
#else
typedef double real;
#define RSQRT sqrt
#endif
#define RL(x) ((real) (x))

struct hcfd_oracle {
    int Nn, Nc, Nf, Ncol, NBC, F_BC, nreal;
    double gma;
    int* coltag; int* coloff;
    double* nodes;
    int* fn_con; int* fc_con; int* cn_off; int* cn_con;
    /* Domain (src/Base/Domain.cpp) */
    double* rf;   /* [Nf][2][2] */
    double* xf;   /* [Nf][2]    */
    double* nf;   /* [Nf][2]    */
    double* Af; double* If;
    double* xc;   /* [Nc][2]    */
    double* iv;
    /* the geometry in the step's arithmetic (the arrays above in the double build) */
    real* rfR; real* nfR; real* AfR; real* IfR; real* ivR;
    /* Euler state (src/Base/Euler.cpp:9-15) */
    real* U[NV]; real* Q[NV]; real* R[NV]; real* phi[NV]; real* G[NV];
    real* Rc[NV];  /* compensation terms of the two-sums (float build) */
    real* Umin; real* Umax; real* dL; real* dR;
    real* dtloc;
    /* BCs */
    int* bc_type; int* bc_F1; int* bc_F2;
    double (*QBC)[NV]; double (*UBC)[NV];
    int limiter; double K;
    long long nsteps, freeze_after;
};

static inline double dot2(const double* a, const double* b) { return a[0]*b[0] + a[1]*b[1]; }
static inline real dot2r(const real* a, const real* b) { return a[0]*b[0] + a[1]*b[1]; }

/* HCFD_ORACLE_NOCOMP (float build only): plain float sums instead of two-sums, to measure what
 * the compensation buys. */
#if defined(HCFD_ORACLE_FP32) && !defined(HCFD_ORACLE_NOCOMP)
#define HCFD_ORACLE_COMP 1
#endif

#ifdef HCFD_ORACLE_COMP
/* s + c += x (Knuth's two-sum); the library's FP32 path accumulates each cell's residual so. */
static inline void two_sum(real* s, real* c, real x) {
    real t = *s + x;
    real bp = t - *s;
    real e = (*s - (t - bp)) + (x - bp);
    *s = t;
    *c += e;
}
#endif

/* Domain::compute_xf / compute_xc / compute_rf / compute_nf / compute_If / compute_iv
 * (src/Base/Domain.cpp:44-146) and zero_bc_iv (:148-154, called by the Euler constructor,
 * src/Base/Euler.cpp:24). */
static void build_domain(hcfd_oracle* o) {
    const int Nf = o->Nf, Nc = o->Nc;
    for (int f = 0; f < Nf; f++) {                                  /* Domain.cpp:44-59 */
        int n1 = o->fn_con[2*f], n2 = o->fn_con[2*f+1];
        for (int d = 0; d < ND; d++)
            o->xf[2*f+d] = 0.5*(o->nodes[ND*n1+d] + o->nodes[ND*n2+d]);
    }
    for (int i = 0; i < Nc; i++) {                                  /* Domain.cpp:61-71 */
        int nnds = o->cn_off[i+1] - o->cn_off[i];
        for (int n = o->cn_off[i]; n < o->cn_off[i+1]; n++) {
            int nd = o->cn_con[n];
            for (int d = 0; d < ND; d++) o->xc[2*i+d] += o->nodes[nd*ND+d]/nnds;
        }
    }
    for (int f = 0; f < Nf; f++) {                                  /* Domain.cpp:73-83 */
        int CL = o->fc_con[2*f], CR = o->fc_con[2*f+1];
        for (int d = 0; d < ND; d++) {
            o->rf[4*f+0+d] = o->xf[2*f+d] - o->xc[2*CL+d];
            o->rf[4*f+2+d] = o->xf[2*f+d] - o->xc[2*CR+d];
        }
    }
    for (int f = o->F_BC; f < Nf; f++)                              /* Domain.cpp:84-88 */
        for (int d = 0; d < ND; d++) o->rf[4*f+2+d] = -o->rf[4*f+0+d];
    for (int f = 0; f < Nf; f++) {                                  /* Domain.cpp:91-116 */
        int n1 = o->fn_con[2*f], n2 = o->fn_con[2*f+1];
        double nd1[ND], nd2[ND];
        for (int d = 0; d < ND; d++) { nd1[d] = o->nodes[ND*n1+d]; nd2[d] = o->nodes[ND*n2+d]; }
        double* n = &o->nf[2*f];
        n[0] =  (nd2[1]-nd1[1]);
        n[1] = -(nd2[0]-nd1[0]);
        o->Af[f] = sqrt(dot2(n, n));
        for (int d = 0; d < ND; d++) n[d] /= o->Af[f];
        double nf_dot_rl = dot2(n, &o->rf[4*f]);
        int sgn = (nf_dot_rl > 0) ? 1 : -1;
        n[0] = sgn*n[0];
        n[1] = sgn*n[1];
    }
    for (int f = 0; f < Nf; f++) {                                  /* Domain.cpp:118-125 */
        double nrL =  dot2(&o->nf[2*f], &o->rf[4*f]);
        double nrR = -dot2(&o->nf[2*f], &o->rf[4*f+2]);
        o->If[f] = nrL/(nrL+nrR);
    }
    for (int f = 0; f < Nf; f++) {                                  /* Domain.cpp:127-136 */
        double AL = o->Af[f]*dot2(&o->nf[2*f], &o->rf[4*f]);
        double AR = o->Af[f]*dot2(&o->nf[2*f], &o->rf[4*f+2]);
        int CL = o->fc_con[2*f], CR = o->fc_con[2*f+1];
        o->iv[CL] += AL/ND;
        o->iv[CR] -= AR/ND;
    }
    for (int i = 0; i < Nc; i++) o->iv[i] = 1.0/o->iv[i];           /* Domain.cpp:138 */
    for (int f = o->F_BC; f < Nf; f++)                              /* Domain.cpp:140-145 */
        o->iv[o->fc_con[2*f+1]] = o->iv[o->fc_con[2*f]];
    for (int f = o->F_BC; f < Nf; f++) o->iv[o->fc_con[2*f+1]] = 0.0; /* Domain.cpp:148-154 */
}

static void* xcalloc(size_t n, size_t sz) { return calloc(n ? n : 1, sz); }

hcfd_oracle* hcfd_oracle_create(int Nn, int Nc, int Nf, int Ncol, int NBCcol,
                                const int* coltag, const int* coloff, const double* nodes,
                                const int* fn_con, const int* fc_con,
                                const int* cn_off, const int* cn_con, double gma) {
    if (Nn <= 0 || Nc <= 0 || Nf <= 0 || Ncol <= 0 || NBCcol < 0 || NBCcol > Ncol) return NULL;
    hcfd_oracle* o = (hcfd_oracle*) xcalloc(1, sizeof(*o));
    o->Nn = Nn; o->Nc = Nc; o->Nf = Nf; o->Ncol = Ncol; o->NBC = NBCcol; o->gma = gma;
    o->coltag = (int*) xcalloc(Ncol, sizeof(int)); memcpy(o->coltag, coltag, sizeof(int)*Ncol);
    o->coloff = (int*) xcalloc(Ncol+1, sizeof(int)); memcpy(o->coloff, coloff, sizeof(int)*(Ncol+1));
    o->F_BC = o->coloff[Ncol-NBCcol];
    o->nodes = (double*) xcalloc((size_t)Nn*ND, sizeof(double)); memcpy(o->nodes, nodes, sizeof(double)*Nn*ND);
    o->fn_con = (int*) xcalloc((size_t)2*Nf, sizeof(int)); memcpy(o->fn_con, fn_con, sizeof(int)*2*Nf);
    o->fc_con = (int*) xcalloc((size_t)2*Nf, sizeof(int)); memcpy(o->fc_con, fc_con, sizeof(int)*2*Nf);
    o->cn_off = (int*) xcalloc(Nc+1, sizeof(int)); memcpy(o->cn_off, cn_off, sizeof(int)*(Nc+1));
    o->cn_con = (int*) xcalloc(cn_off[Nc], sizeof(int)); memcpy(o->cn_con, cn_con, sizeof(int)*cn_off[Nc]);
    o->rf = (double*) xcalloc((size_t)4*Nf, sizeof(double));
    o->xf = (double*) xcalloc((size_t)2*Nf, sizeof(double));
    o->nf = (double*) xcalloc((size_t)2*Nf, sizeof(double));
    o->Af = (double*) xcalloc(Nf, sizeof(double));
    o->If = (double*) xcalloc(Nf, sizeof(double));
    o->xc = (double*) xcalloc((size_t)2*Nc, sizeof(double));
    o->iv = (double*) xcalloc(Nc, sizeof(double));
    for (int v = 0; v < NV; v++) {
        o->U[v] = (real*) xcalloc(Nc, sizeof(real));
        o->Q[v] = (real*) xcalloc(Nc, sizeof(real));
        o->R[v] = (real*) xcalloc(Nc, sizeof(real));
        o->Rc[v] = (real*) xcalloc(Nc, sizeof(real));
        o->phi[v] = (real*) xcalloc(Nc, sizeof(real));
        o->G[v] = (real*) xcalloc((size_t)2*Nc, sizeof(real));
    }
    o->Umin = (real*) xcalloc(Nc, sizeof(real));
    o->Umax = (real*) xcalloc(Nc, sizeof(real));
    o->dL = (real*) xcalloc(Nf, sizeof(real));
    o->dR = (real*) xcalloc(Nf, sizeof(real));
    o->dtloc = (real*) xcalloc(Nc, sizeof(real));
    o->bc_type = (int*) xcalloc(NBCcol, sizeof(int));
    o->bc_F1 = (int*) xcalloc(NBCcol, sizeof(int));
    o->bc_F2 = (int*) xcalloc(NBCcol, sizeof(int));
    o->QBC = (double (*)[NV]) xcalloc(NBCcol, sizeof(double[NV]));
    o->UBC = (double (*)[NV]) xcalloc(NBCcol, sizeof(double[NV]));
    build_domain(o);
#ifdef HCFD_ORACLE_FP32
    o->rfR = (real*) xcalloc((size_t)4*Nf, sizeof(real));
    o->nfR = (real*) xcalloc((size_t)2*Nf, sizeof(real));
    o->AfR = (real*) xcalloc(Nf, sizeof(real));
    o->IfR = (real*) xcalloc(Nf, sizeof(real));
    o->ivR = (real*) xcalloc(Nc, sizeof(real));
    for (size_t k = 0; k < (size_t)4*Nf; k++) o->rfR[k] = RL(o->rf[k]);
    for (size_t k = 0; k < (size_t)2*Nf; k++) o->nfR[k] = RL(o->nf[k]);
    for (int f = 0; f < Nf; f++) { o->AfR[f] = RL(o->Af[f]); o->IfR[f] = RL(o->If[f]); }
    for (int i = 0; i < Nc; i++) o->ivR[i] = RL(o->iv[i]);
#else
    o->rfR = o->rf; o->nfR = o->nf; o->AfR = o->Af; o->IfR = o->If; o->ivR = o->iv;
#endif
    o->nreal = 0;
    for (int i = 0; i < Nc; i++) o->nreal += (o->iv[i] != 0.0);
    return o;
}

void hcfd_oracle_free(hcfd_oracle* o) {
    if (!o) return;
    free(o->coltag); free(o->coloff); free(o->nodes); free(o->fn_con); free(o->fc_con);
    free(o->cn_off); free(o->cn_con); free(o->rf); free(o->xf); free(o->nf); free(o->Af);
    free(o->If); free(o->xc); free(o->iv);
    for (int v = 0; v < NV; v++) {
        free(o->U[v]); free(o->Q[v]); free(o->R[v]); free(o->Rc[v]); free(o->phi[v]); free(o->G[v]);
    }
#ifdef HCFD_ORACLE_FP32
    free(o->rfR); free(o->nfR); free(o->AfR); free(o->IfR); free(o->ivR);
#endif
    free(o->Umin); free(o->Umax); free(o->dL); free(o->dR); free(o->dtloc);
    free(o->bc_type); free(o->bc_F1); free(o->bc_F2); free(o->QBC); free(o->UBC);
    free(o);
}

int hcfd_oracle_nreal(hcfd_oracle* o) { return o->nreal; }

/* Primitive -> conservative, BoundaryCondition::init (src/Base/BoundaryConditions/Base.cpp:18-22)
 * and Euler::initialise (src/Base/Euler.cpp:63-68). */
static void prim_to_cons(const double* q, double gma, double* u) {
    u[0] = q[0];
    for (int v = 1; v < NV; v++) u[v] = q[0]*q[v];
    u[ND+1] = q[ND+1]/(gma-1) + 0.5*q[0]*dot2(&q[1], &q[1]);
}

int hcfd_oracle_gather_bcs(hcfd_oracle* o, const int* bcmap, int nbcmap, const double* qbc) {
    int fcolBC = o->Ncol - o->NBC;                                  /* Euler.cpp:43-59 */
    for (int fcol = fcolBC; fcol < o->Ncol; fcol++) {
        int bc = fcol - fcolBC;
        int tag = o->coltag[fcol];
        if (tag < 0 || tag >= nbcmap) return -1;
        int t = bcmap[tag];
        if (t < 0 || t > 5) return -1;
        o->bc_type[bc] = t;
        o->bc_F1[bc] = o->coloff[fcol];
        o->bc_F2[bc] = o->coloff[fcol+1];
        for (int v = 0; v < NV; v++) o->QBC[bc][v] = qbc[NV*bc+v];
        prim_to_cons(o->QBC[bc], o->gma, o->UBC[bc]);
    }
    return 0;
}

/* update_cells of each BC type, in BC order (src/Base/Euler.cpp:138-142). */
static void update_bc_cells(hcfd_oracle* o) {
    real** U = o->U;
    const double gma = o->gma;
    for (int bc = 0; bc < o->NBC; bc++) {
        for (int f = o->bc_F1[bc]; f < o->bc_F2[bc]; f++) {
            int CL = o->fc_con[2*f], CR = o->fc_con[2*f+1];
            switch (o->bc_type[bc]) {
            case 0: {                                   /* Symmetry.cpp:5-24 */
                const real* n = &o->nfR[2*f];
                real ul[ND];
                for (int d = 0; d < ND; d++) ul[d] = U[d+1][CL];
                real nor = dot2r(ul, n);
                U[0][CR] = U[0][CL];
                for (int d = 0; d < ND; d++) U[d+1][CR] = ul[d] - 2*nor*n[d];
                U[ND+1][CR] = U[ND+1][CL];
            } break;
            case 1:                                     /* Wall.cpp:4-15 */
                U[0][CR] = U[0][CL];
                for (int v = 1; v < ND+1; v++) U[v][CR] = -U[v][CL];
                U[ND+1][CR] = U[ND+1][CL];
                break;
            case 2:                                     /* Inlet.cpp:4-13 */
                for (int v = 0; v < NV; v++) U[v][CR] = RL(o->UBC[bc][v]);
                break;
            case 3: {                                   /* Inlet.cpp:15-31 */
                real UL[NV];
                for (int v = 0; v < NV; v++) UL[v] = U[v][CL];
                real PL = RL(gma-1)*(UL[ND+1] - RL(0.5)*dot2r(&UL[1], &UL[1])/UL[0]);
                for (int v = 0; v < NV; v++) U[v][CR] = RL(o->UBC[bc][v]);
                U[ND+1][CR] = PL/RL(gma-1) + RL(0.5*o->QBC[bc][0]*dot2(&o->QBC[bc][1], &o->QBC[bc][1]));
            } break;
            case 4:                                     /* Outlet.cpp:4-13 */
                for (int v = 0; v < NV; v++) U[v][CR] = U[v][CL];
                break;
            case 5: {                                   /* Outlet.cpp:15-32, as intended */
                /* The reference's loop (Outlet.cpp:26-28) reads rul[-1] (undefined) and
                 * stops one momentum component short.  Restated as a subsonic outlet that
                 * takes rho and rho*u from the interior and p from the BC state. */
                real rl = U[0][CL];
                real rul[ND];
                for (int d = 0; d < ND; d++) rul[d] = U[d+1][CL];
                U[0][CR] = rl;
                for (int d = 0; d < ND; d++) U[d+1][CR] = rul[d];
                U[ND+1][CR] = RL(o->QBC[bc][ND+1]/(gma-1)) + RL(0.5)*dot2r(rul, rul)/rl;
            } break;
            }
        }
    }
}

int hcfd_oracle_initialise(hcfd_oracle* o, const double* qic) {
    double UIC[NV];
    prim_to_cons(qic, o->gma, UIC);
    for (int v = 0; v < NV; v++)
        for (int i = 0; i < o->Nc; i++) o->U[v][i] = RL(UIC[v]);
    update_bc_cells(o);
    o->nsteps = 0;
    return 0;
}

/* Limiter freezing (not in the reference): steps 1..after compute the limiter as usual; every
 * later step reuses the limiter values of step `after` with fresh gradients.  0 = never. */
int hcfd_oracle_set_freeze(hcfd_oracle* o, long long after) {
    if (after < 0) return -1;
    o->freeze_after = after;
    return 0;
}

int hcfd_oracle_set_limiter(hcfd_oracle* o, int kind, double K) {
    if (kind != HCFD_OR_BJ && kind != HCFD_OR_VENKAT) return -1;
    o->limiter = kind; o->K = K;
    return 0;
}

/* GaussGreen::compute_gradient (src/Base/GaussGreen.cpp:14-40). */
static void gradient(hcfd_oracle* o) {
    const int Nc = o->Nc, Nf = o->Nf;
    for (int v = 0; v < NV; v++) memset(o->G[v], 0, sizeof(real)*2*Nc);
    for (int f = 0; f < Nf; f++) {
        int CL = o->fc_con[2*f], CR = o->fc_con[2*f+1];
        for (int v = 0; v < NV; v++) {
            for (int d = 0; d < ND; d++) {
                real uf = o->U[v][CL]*o->IfR[f] + o->U[v][CR]*(1-o->IfR[f]);
                o->G[v][d*Nc+CL] += uf*o->AfR[f]*o->nfR[2*f+d];
                o->G[v][d*Nc+CR] -= uf*o->AfR[f]*o->nfR[2*f+d];
            }
        }
    }
    for (int v = 0; v < NV; v++)
        for (int d = 0; d < ND; d++)
            for (int i = 0; i < Nc; i++) o->G[v][d*Nc+i] *= o->ivR[i];
}

/* One side of a face for the Venkatakrishnan limiter: d = grad.r, D1 = Umax-U or Umin-U,
 * eps2 = (K h)^3 with h = sqrt(cell area).
 *   phi = min(1, (D1^2 + eps2 + 2 D1 d) / (D1^2 + 2 d^2 + D1 d + eps2)). */
static inline real venkat(real D1, real d, real eps2) {
    real num = D1*D1 + eps2 + RL(2)*D1*d;
    real den = D1*D1 + RL(2)*d*d + D1*d + eps2;
    return fmin(1, num/den);
}

/* Limiter::limit_gradient (src/Base/Limiter.cpp:19-77); the Venkatakrishnan branch replaces
 * the Barth-Jespersen ratio with venkat() and keeps everything else. */
static void limiter(hcfd_oracle* o) {
    const real eps = RL(1e-9);
    const int Nf = o->Nf, Nc = o->Nc;
    real GL[ND], GR[ND];
    for (int v = 0; v < NV; v++) {
        memcpy(o->Umin, o->U[v], Nc*sizeof(real));
        memcpy(o->Umax, o->U[v], Nc*sizeof(real));
        for (int i = 0; i < Nc; i++) o->phi[v][i] = 1.0;
        for (int f = 0; f < Nf; f++) {
            int CL = o->fc_con[2*f], CR = o->fc_con[2*f+1];
            o->Umin[CL] = fmin(o->Umin[CL], o->U[v][CR]);
            o->Umax[CL] = fmax(o->Umax[CL], o->U[v][CR]);
            o->Umin[CR] = fmin(o->Umin[CR], o->U[v][CL]);
            o->Umax[CR] = fmax(o->Umax[CR], o->U[v][CL]);
        }
        for (int f = 0; f < Nf; f++) {
            int CL = o->fc_con[2*f], CR = o->fc_con[2*f+1];
            for (int d = 0; d < ND; d++) { GL[d] = o->G[v][d*Nc+CL]; GR[d] = o->G[v][d*Nc+CR]; }
            o->dL[f] = dot2r(GL, &o->rfR[4*f]);
            o->dR[f] = dot2r(GR, &o->rfR[4*f+2]);
        }
        for (int f = 0; f < Nf; f++) {
            int CL = o->fc_con[2*f], CR = o->fc_con[2*f+1];
            real UL = o->U[v][CL], UR = o->U[v][CR];
            real phi_fl = 1.0, phi_fr = 1.0;
            real dLf = o->dL[f], dRf = o->dR[f];
            if (o->limiter == HCFD_OR_BJ) {
                phi_fl = (dLf >  eps) ? fmin(1, (o->Umax[CL]-UL)/dLf) : phi_fl;
                phi_fl = (dLf < -eps) ? fmin(1, (o->Umin[CL]-UL)/dLf) : phi_fl;
                phi_fr = (dRf >  eps) ? fmin(1, (o->Umax[CR]-UR)/dRf) : phi_fr;
                phi_fr = (dRf < -eps) ? fmin(1, (o->Umin[CR]-UR)/dRf) : phi_fr;
            } else {
                real kL = o->ivR[CL] != 0 ? RL(o->K)*RSQRT(RL(1.0)/o->ivR[CL]) : RL(0.0);
                real kR = o->ivR[CR] != 0 ? RL(o->K)*RSQRT(RL(1.0)/o->ivR[CR]) : RL(0.0);
                real eL = kL*kL*kL, eR = kR*kR*kR;
                phi_fl = (dLf >  eps) ? venkat(o->Umax[CL]-UL, dLf, eL) : phi_fl;
                phi_fl = (dLf < -eps) ? venkat(o->Umin[CL]-UL, dLf, eL) : phi_fl;
                phi_fr = (dRf >  eps) ? venkat(o->Umax[CR]-UR, dRf, eR) : phi_fr;
                phi_fr = (dRf < -eps) ? venkat(o->Umin[CR]-UR, dRf, eR) : phi_fr;
            }
            o->phi[v][CL] = fmin(o->phi[v][CL], phi_fl);
            o->phi[v][CR] = fmin(o->phi[v][CR], phi_fr);
        }
    }
}

/* BoundaryCondition::update_grads / update_limiter (src/Base/BoundaryConditions/Base.cpp:29-53). */
static void bc_grads_limiter(hcfd_oracle* o) {
    const int Nc = o->Nc;
    for (int bc = 0; bc < o->NBC; bc++) {
        for (int v = 0; v < NV; v++)
            for (int d = 0; d < ND; d++)
                for (int f = o->bc_F1[bc]; f < o->bc_F2[bc]; f++) {
                    int CL = o->fc_con[2*f], CR = o->fc_con[2*f+1];
                    o->G[v][d*Nc+CR] = -o->G[v][d*Nc+CL];
                }
        for (int v = 0; v < NV; v++)
            for (int f = o->bc_F1[bc]; f < o->bc_F2[bc]; f++) {
                int CL = o->fc_con[2*f], CR = o->fc_con[2*f+1];
                o->phi[v][CR] = o->phi[v][CL];
            }
    }
}

/* Flux::EulerFlux (src/Base/Flux.cpp:89-97). */
static inline void euler_flux(const real U[NV], const real n[ND], real gma, real F[NV]) {
    real gmo = gma-1;
    real ir = RL(1.0)/U[0];
    real P = gmo* (U[ND+1] - RL(0.5)*ir*dot2r(&U[1],&U[1]));
    F[0] = n[0]* U[1]              + n[1]* U[2]             ;
    F[1] = n[0]*(U[1]*U[1]*ir + P) + n[1]* U[2]*U[1]*ir     ;
    F[2] = n[0]* U[1]*U[2]*ir      + n[1]*(U[2]*U[2]*ir + P);
    F[3] = n[0]*(U[3]+P)*U[1]*ir   + n[1]*(U[3]+P)*U[2]*ir  ;
}

/* Flux::Rusanov (src/Base/Flux.cpp:52-81). */
static inline void rusanov(const real UL[NV], const real UR[NV], const real n[ND],
                           real gma, real F[NV]) {
    real gmo = gma-1;
    real irl = RL(1.0)/UL[0];
    real irr = RL(1.0)/UR[0];
    real nvl = dot2r(n, &UL[1])*irl;
    real nvr = dot2r(n, &UR[1])*irr;
    real qql = RL(0.5)*dot2r(&UL[1], &UL[1])*irl;
    real qqr = RL(0.5)*dot2r(&UR[1], &UR[1])*irr;
    real pl  = gmo*(UL[ND+1] - qql);
    real pr  = gmo*(UR[ND+1] - qqr);
    real al  = RSQRT(gma*pl*irl);
    real ar  = RSQRT(gma*pr*irr);
    real S1  = fmax(fabs(nvl-al), fabs(nvr-ar));
    real S2  = fmax(fabs(nvl+al), fabs(nvr+ar));
    real S   = fmax(S1, S2);
    real FL[NV], FR[NV];
    euler_flux(UL, n, gma, FL);
    euler_flux(UR, n, gma, FR);
    for (int v = 0; v < NV; v++) F[v] = RL(0.5) * ( (FL[v] + FR[v]) - S*(UR[v] - UL[v]) );
}

/* Flux::ComputeFlux with Flux::MUSCL (src/Base/Flux.cpp:9-50, 83-87). */
static void flux(hcfd_oracle* o) {
    const int Nc = o->Nc, Nf = o->Nf;
    real UL[NV], UR[NV], phiL[NV], phiR[NV], GL[NV][ND], GR[NV][ND];
    real UfL[NV], UfR[NV], Ff[NV];
    for (int f = 0; f < Nf; f++) {
        int CL = o->fc_con[2*f], CR = o->fc_con[2*f+1];
        real Af = o->AfR[f];
        for (int v = 0; v < NV; v++) {
            UL[v] = o->U[v][CL]; UR[v] = o->U[v][CR];
            phiL[v] = o->phi[v][CL]; phiR[v] = o->phi[v][CR];
            for (int d = 0; d < ND; d++) { GL[v][d] = o->G[v][d*Nc+CL]; GR[v][d] = o->G[v][d*Nc+CR]; }
        }
        const real* rL = &o->rfR[4*f];
        const real* rR = &o->rfR[4*f+2];
        for (int v = 0; v < NV; v++) UfL[v] = UL[v] + phiL[v]*dot2r(GL[v], rL);
        for (int v = 0; v < NV; v++) UfR[v] = UR[v] + phiR[v]*dot2r(GR[v], rR);
        rusanov(UfL, UfR, &o->nfR[2*f], RL(o->gma), Ff);
        for (int v = 0; v < NV; v++) {
#ifdef HCFD_ORACLE_COMP
            two_sum(&o->R[v][CL], &o->Rc[v][CL], -(Af*Ff[v]));
            two_sum(&o->R[v][CR], &o->Rc[v][CR], Af*Ff[v]);
#else
            o->R[v][CL] -= Af*Ff[v];
            o->R[v][CR] += Af*Ff[v];
#endif
        }
    }
#ifdef HCFD_ORACLE_COMP
    for (int v = 0; v < NV; v++)
        for (int i = 0; i < Nc; i++) { o->R[v][i] = (o->R[v][i] + o->Rc[v][i])*o->ivR[i]; o->Rc[v][i] = 0; }
#else
    for (int v = 0; v < NV; v++)
        for (int i = 0; i < Nc; i++) o->R[v][i] *= o->ivR[i];
#endif
}

/* Local time step at CFL 1 for each real cell c (iv_c != 0):
 *   lam_c = sum over the faces of c, in increasing face order, of (|u_c.n_f| + a_c) A_f
 *   dt_c  = 1 / (iv_c lam_c)
 * with u_c = (rho u, rho v)/rho and a_c = sqrt(gma p_c / rho_c) from the cell's own state.
 * Ghost cells get 0.  Faces are visited in increasing index, as in the reference's
 * cell->face table (src/Mesh.cpp:88-117). */
static void local_dt(hcfd_oracle* o) {
    const int Nc = o->Nc, Nf = o->Nf;
    const real gma = RL(o->gma);
    const real gmo = gma - 1;
    real* lam = o->dtloc;
    memset(lam, 0, sizeof(real)*Nc);
    for (int f = 0; f < Nf; f++) {
        int C2[2] = { o->fc_con[2*f], o->fc_con[2*f+1] };
        for (int s = 0; s < 2; s++) {
            int c = C2[s];
            if (o->iv[c] == 0.0) continue;
            real ir = RL(1.0)/o->U[0][c];
            real u = o->U[1][c]*ir, v = o->U[2][c]*ir;
            real p = gmo*(o->U[3][c] - RL(0.5)*(o->U[1][c]*u + o->U[2][c]*v));
            real a = RSQRT(gma*p*ir);
            real un = u*o->nfR[2*f] + v*o->nfR[2*f+1];
            lam[c] += (fabs(un) + a)*o->AfR[f];
        }
    }
    for (int i = 0; i < Nc; i++) lam[i] = (o->iv[i] != 0.0) ? RL(1.0)/(o->ivR[i]*lam[i]) : RL(0.0);
}

int hcfd_oracle_phase(hcfd_oracle* o, int which, double dt) {
    switch (which) {
    case 0: gradient(o); break;
    case 1: limiter(o); break;
    case 2: bc_grads_limiter(o); break;
    case 3: flux(o); break;
    case 4:
        for (int v = 0; v < NV; v++)
            for (int i = 0; i < o->Nc; i++) o->U[v][i] += RL(dt)*o->R[v][i];   /* Euler.cpp:107-113 */
        break;
    case 5: for (int v = 0; v < NV; v++) memset(o->R[v], 0, sizeof(real)*o->Nc); break;
    case 6: update_bc_cells(o); break;
    default: return -1;
    }
    return 0;
}

/* One loop iteration of Euler::run (src/Base/Euler.cpp:86-96) with the dt choice widened. */
int hcfd_oracle_step(hcfd_oracle* o, int mode, double dt_or_cfl, double* dt_used, double* res_l2) {
    const int Nc = o->Nc;
    double dt = dt_or_cfl;
    if (mode != HCFD_OR_FIXED_DT) {
        local_dt(o);
        double mn = INFINITY;
        for (int i = 0; i < Nc; i++) if (o->iv[i] != 0.0 && o->dtloc[i] < mn) mn = o->dtloc[i];
        dt = dt_or_cfl*mn;
        if (mode == HCFD_OR_LOCAL_CFL)
            for (int i = 0; i < Nc; i++) o->dtloc[i] *= RL(dt_or_cfl);
    }
    gradient(o);
    o->nsteps++;
    if (o->freeze_after <= 0 || o->nsteps <= o->freeze_after) limiter(o);
    bc_grads_limiter(o);
    flux(o);
    if (res_l2) {
        double s = 0.0;
        for (int i = 0; i < Nc; i++) if (o->iv[i] != 0.0) s += (double) o->R[0][i]*(double) o->R[0][i];
        *res_l2 = sqrt(s/o->nreal);
    }
    if (mode == HCFD_OR_LOCAL_CFL) {
        for (int v = 0; v < NV; v++)
            for (int i = 0; i < Nc; i++) o->U[v][i] += o->dtloc[i]*o->R[v][i];
    } else {
        for (int v = 0; v < NV; v++)
            for (int i = 0; i < Nc; i++) o->U[v][i] += RL(dt)*o->R[v][i];
    }
    for (int v = 0; v < NV; v++) memset(o->R[v], 0, sizeof(real)*Nc);
    update_bc_cells(o);
    if (dt_used) *dt_used = dt;
    return 0;
}

/* Euler::compute_prims (src/Base/Euler.cpp:115-136). */
static void prims(hcfd_oracle* o) {
    const int Nc = o->Nc;
    for (int i = 0; i < Nc; i++) o->Q[0][i] = o->U[0][i];
    for (int v = 1; v < NV; v++) {
        if (v == ND+1) continue;
        for (int i = 0; i < Nc; i++) o->Q[v][i] = o->U[v][i]/o->U[0][i];
    }
    real gmo = RL(o->gma)-1;
    for (int i = 0; i < Nc; i++) {
        real u[ND];
        for (int d = 0; d < ND; d++) u[d] = o->Q[d+1][i];
        o->Q[ND+1][i] = gmo * (o->U[ND+1][i] - RL(0.5)*o->Q[0][i]*dot2r(u,u));
    }
}

static void widen(double* out, const real* in, size_t n) { for (size_t k = 0; k < n; k++) out[k] = in[k]; }
static void narrow(real* out, const double* in, size_t n) { for (size_t k = 0; k < n; k++) out[k] = RL(in[k]); }

int hcfd_oracle_get(hcfd_oracle* o, int which, double* out) {
    const int Nc = o->Nc;
    switch (which) {
    case HCFD_OR_U: for (int v = 0; v < NV; v++) widen(out + (size_t)v*Nc, o->U[v], Nc); break;
    case HCFD_OR_Q: prims(o); for (int v = 0; v < NV; v++) widen(out + (size_t)v*Nc, o->Q[v], Nc); break;
    case HCFD_OR_PHI: for (int v = 0; v < NV; v++) widen(out + (size_t)v*Nc, o->phi[v], Nc); break;
    case HCFD_OR_R: for (int v = 0; v < NV; v++) widen(out + (size_t)v*Nc, o->R[v], Nc); break;
    case HCFD_OR_G: for (int v = 0; v < NV; v++) widen(out + (size_t)v*2*Nc, o->G[v], (size_t)2*Nc); break;
    case HCFD_OR_DTLOC: local_dt(o); widen(out, o->dtloc, Nc); break;
    case HCFD_OR_IV: memcpy(out, o->iv, sizeof(double)*Nc); break;
    default: return -1;
    }
    return 0;
}

/* Replaces the state (rounded to the step's arithmetic). */
int hcfd_oracle_set_U(hcfd_oracle* o, const double* u) {
    for (int v = 0; v < NV; v++) narrow(o->U[v], u + (size_t)v*o->Nc, o->Nc);
    return 0;
}

/* Replaces the limiter values (used by the next steps only while the limiter is frozen; an
 * unfrozen step recomputes them). */
int hcfd_oracle_set_phi(hcfd_oracle* o, const double* phi) {
    for (int v = 0; v < NV; v++) narrow(o->phi[v], phi + (size_t)v*o->Nc, o->Nc);
    return 0;
}

int hcfd_oracle_wall_cp(hcfd_oracle* o, int colour, double rho_inf, double p_inf,
                        double speed_inf, double* out) {
    if (colour < 0 || colour >= o->Ncol) return -1;
    const double gmo = o->gma - 1;
    const double qinf = 0.5*rho_inf*speed_inf*speed_inf;
    int k = 0;
    for (int f = o->coloff[colour]; f < o->coloff[colour+1]; f++) {
        int c = o->fc_con[2*f];
        double r = o->U[0][c], ru = o->U[1][c], rv = o->U[2][c], E = o->U[3][c];
        double p = gmo*(E - 0.5*(ru*ru + rv*rv)/r);
        out[k++] = (p - p_inf)/qinf;
    }
    return k;
}

int hcfd_oracle_domain(hcfd_oracle* o, double* rf, double* nf, double* Af, double* If,
                       double* xc, double* iv) {
    memcpy(rf, o->rf, sizeof(double)*4*o->Nf);
    memcpy(nf, o->nf, sizeof(double)*2*o->Nf);
    memcpy(Af, o->Af, sizeof(double)*o->Nf);
    memcpy(If, o->If, sizeof(double)*o->Nf);
    memcpy(xc, o->xc, sizeof(double)*2*o->Nc);
    memcpy(iv, o->iv, sizeof(double)*o->Nc);
    return 0;
}
