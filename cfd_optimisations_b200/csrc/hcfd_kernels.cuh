// Device kernels of the B200 solver: geometry precompute, the two fused step passes, the
// ghost-cell refresh, and the conversions in and out of the device state.
//
// Step structure (one time step = two launches, no atomics on the data path):
//   pass 1 (cell-centric): Green-Gauss gradient, Barth-Jespersen / Venkatakrishnan limiter,
//     and (CFL modes) the cell's local dt folded into a grid-wide minimum.  Writes
//     phiG = phi * grad U per cell (the limited gradient, 8 values).
//   pass 2 (cell-centric): MUSCL face states on both sides, Rusanov flux, signed gather of
//     the face fluxes in increasing face order, U += dt R, and the refresh of the cell's own
//     ghost cells; residual norm folded into a deterministic two-level reduction.
// The reference runs the same arithmetic as face loops that scatter into both cells
// (src/Base/GaussGreen.cpp:19-31, Limiter.cpp:26-76, Flux.cpp:19-43); here each cell
// gathers over its faces in increasing face index, which is the order in which the
// reference's scatter adds into that cell, so every per-cell sum is formed in the
// reference's order and the result does not depend on thread scheduling.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace hcfd {

constexpr int NV = 4;
constexpr int MAXBC = 16;

enum { LIM_BJ = 0, LIM_VENKAT = 1 };
enum { TM_FIXED = 0, TM_GLOBAL = 1, TM_LOCAL = 2 };

// Face record: unit normal (oriented out of CL), length, interpolation weight and the two
// centre-to-face vectors (includes/Base/Domain.hpp:15-20).  64 B in double, 32 B in float.
template <class T>
struct alignas(8 * sizeof(T)) FaceGeo {
    T nx, ny, Af, If, rLx, rLy, rRx, rRy;
};

// Conserved state of one cell, (rho, rho u, rho v, E): 32 B in double, 16 B in float.
template <class T>
struct alignas(4 * sizeof(T)) Cell4 {
    T v[4];
};

// Limited gradient phi_v * dU_v/dx_d of one cell, [v][d].
template <class T>
struct alignas(8 * sizeof(T)) Grad8 {
    T g[8];
};

struct BCTable {
    int nbc;
    int F1[MAXBC + 1];       // first face of BC k; F1[nbc] = Nf
    int type[MAXBC];
    double UBC[MAXBC][4];    // conservative BC state (BoundaryCondition::init)
    double QBC[MAXBC][4];    // primitive BC state
};

// Small device-side record of the step history (read by the host on demand).
struct StepStats {
    double res2_last;        // sum over real cells of R_rho^2, last step
    double res2_first;       // same, first step since initialise
    double dt_last;          // dt of the last step (min local dt under local stepping)
    long long steps;         // steps since initialise
    int nonfinite;           // sticky: a step produced a NaN/Inf
    int pad;
};

// Checked build (HCFD_CHECKED, lib/libhcfd_gpu_checked.so): every index the step kernels take
// from their tables is range-checked on the device before it is used, and a violation sets
// bit 2 of the error word (the host reports HCFD_EINVAL).  The tiled kernels check their
// plan's indices (tile descriptors, halo ids, cell slots, entry metadata) where they read
// them, replacing a bad one by an index in range or skipping the access; the per-cell
// kernels' slot table is checked by check_slots_kernel before a step, and no step is launched
// on a bad one.  The default build relies on the host-side checks of every mesh and plan
// (validate_view, the plan builder, hcfd_plan_check) and compiles without the checks.
#ifdef HCFD_CHECKED
constexpr bool kChecked = true;
#else
constexpr bool kChecked = false;
#endif
__device__ __forceinline__ bool index_ok(bool ok, unsigned int* err) {
    if (kChecked && !ok) atomicOr(err, 4u);
    return !kChecked || ok;
}
template <class T>
struct StepArgs {
    const Cell4<T>* __restrict__ U;      // state at step start
    Cell4<T>* __restrict__ Unew;         // state at step end (pass 2)
    Grad8<T>* __restrict__ phiG;         // written by pass 1, read by pass 2
    const FaceGeo<T>* __restrict__ geo;
    const int2* __restrict__ slot;       // [W][Nc]: {face or ~face, neighbour}
    const T* __restrict__ iv;
    unsigned long long* dtmin;           // grid minimum of the CFL-1 local dt (double bits)
    unsigned long long* dtmin_next;      // the other parity slot, reset by pass 2
    double* partial;                     // per-block residual partial sums
    unsigned int* counter;               // blocks done, for the last-block reduction
    StepStats* stats;
    int Nc, F_BC;
    int limiter, time_mode;
    T gma, venkat_K;
    double dt_or_cfl;
    BCTable bc;
    // Limiter freezing: the limiter values of step freeze_after are recorded in phiF and
    // reused by every later step (freeze_after = 0: never).  Steps are counted on the device.
    Cell4<T>* phiF;
    long long freeze_after;
};

enum { LIM_NORMAL = 0, LIM_RECORD = 1, LIM_FROZEN = 2 };
// How pass 1 treats the limiter in the step after `steps_before` steps.
__device__ __forceinline__ int limiter_mode(long long steps_before, long long freeze_after) {
    if (freeze_after <= 0 || steps_before + 1 < freeze_after) return LIM_NORMAL;
    return steps_before + 1 == freeze_after ? LIM_RECORD : LIM_FROZEN;
}

// ---------------------------------------------------------------------------------------
// loads

// Per-cell records (the state Cell4 and the limited gradient Grad8) are stored as 16-byte
// chunk planes: chunk j of record i sits at byte (j * ps + i) * 16 from the base, ps being the
// plane stride in chunks (Nc in HBM, the staged cell count in shared memory).  Random
// 16-byte gathers then spread over all shared-memory bank groups, and a warp's accesses to
// consecutive records are contiguous in every plane.  Cell4: 2 chunks in double, 1 in
// float; Grad8: 4 and 2.
__device__ __forceinline__ void ld_cell(const Cell4<double>* p, size_t ps, int i, double u[4]) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = __ldg(q + i), b = __ldg(q + ps + i);
    u[0] = a.x; u[1] = a.y; u[2] = b.x; u[3] = b.y;
}
__device__ __forceinline__ void ld_cell(const Cell4<float>* p, size_t, int i, float u[4]) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p) + i);
    u[0] = a.x; u[1] = a.y; u[2] = a.z; u[3] = a.w;
}
__device__ __forceinline__ void st_cell(Cell4<double>* p, size_t ps, int i, const double u[4]) {
    double2* q = reinterpret_cast<double2*>(p);
    q[i] = make_double2(u[0], u[1]);
    q[ps + i] = make_double2(u[2], u[3]);
}
__device__ __forceinline__ void st_cell(Cell4<float>* p, size_t, int i, const float u[4]) {
    reinterpret_cast<float4*>(p)[i] = make_float4(u[0], u[1], u[2], u[3]);
}
__device__ __forceinline__ void ld_geo(const FaceGeo<double>* p, int f, FaceGeo<double>& g) {
    const double2* q = reinterpret_cast<const double2*>(p + f);
    double2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3);
    g.nx = a.x; g.ny = a.y; g.Af = b.x; g.If = b.y; g.rLx = c.x; g.rLy = c.y; g.rRx = d.x; g.rRy = d.y;
}
__device__ __forceinline__ void ld_geo(const FaceGeo<float>* p, int f, FaceGeo<float>& g) {
    const float4* q = reinterpret_cast<const float4*>(p + f);
    float4 a = __ldg(q), b = __ldg(q + 1);
    g.nx = a.x; g.ny = a.y; g.Af = a.z; g.If = a.w; g.rLx = b.x; g.rLy = b.y; g.rRx = b.z; g.rRy = b.w;
}
__device__ __forceinline__ void ld_grad(const Grad8<double>* p, size_t ps, int i, double g[8]) {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int k = 0; k < 4; k++) { const double2 a = __ldg(q + k * ps + i); g[2 * k] = a.x; g[2 * k + 1] = a.y; }
}
__device__ __forceinline__ void ld_grad(const Grad8<float>* p, size_t ps, int i, float g[8]) {
    const float4* q = reinterpret_cast<const float4*>(p);
    const float4 a = __ldg(q + i), b = __ldg(q + ps + i);
    g[0] = a.x; g[1] = a.y; g[2] = a.z; g[3] = a.w; g[4] = b.x; g[5] = b.y; g[6] = b.z; g[7] = b.w;
}
__device__ __forceinline__ void st_grad(Grad8<double>* p, size_t ps, int i, const double g[8]) {
    double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
    for (int k = 0; k < 4; k++) q[k * ps + i] = make_double2(g[2 * k], g[2 * k + 1]);
}
__device__ __forceinline__ void st_grad(Grad8<float>* p, size_t ps, int i, const float g[8]) {
    float4* q = reinterpret_cast<float4*>(p);
    q[i] = make_float4(g[0], g[1], g[2], g[3]);
    q[ps + i] = make_float4(g[4], g[5], g[6], g[7]);
}

// ---------------------------------------------------------------------------------------
// Reciprocals, quotients and square roots of the step arithmetic.  FP64 keeps the IEEE
// operations (bit parity with the reference needs them); FP32 uses the hardware
// approximations (a few units in the last place), since nothing compares FP32 bit for bit and
// the IEEE sequences would cost a fair share of the FP32 kernels' issue slots.
template <class T>
__device__ __forceinline__ T qrcp(T x) { return T(1) / x; }
template <>
__device__ __forceinline__ float qrcp<float>(float x) { return __fdividef(1.0f, x); }
template <class T>
__device__ __forceinline__ T qdiv(T a, T b) { return a / b; }
template <>
__device__ __forceinline__ float qdiv<float>(float a, float b) { return __fdividef(a, b); }
template <class T>
__device__ __forceinline__ T qsqrt(T x) { return sqrt(x); }
template <>
__device__ __forceinline__ float qsqrt<float>(float x) { return x == 0.0f ? 0.0f : x * rsqrtf(x); }

// ---------------------------------------------------------------------------------------
// flux arithmetic, written with the reference's expression trees

// Flux::EulerFlux (src/Base/Flux.cpp:89-97); ir = 1/U[0], which Rusanov has formed already
// (the same IEEE quotient, so passing it on changes no bit).
template <class T>
__device__ __forceinline__ void euler_flux(const T U[4], T ir, T n0, T n1, T gma, T F[4]) {
    const T gmo = gma - T(1);
    const T P = gmo * (U[3] - T(0.5) * ir * (U[1] * U[1] + U[2] * U[2]));
    F[0] = n0 * U[1] + n1 * U[2];
    F[1] = n0 * (U[1] * U[1] * ir + P) + n1 * U[2] * U[1] * ir;
    F[2] = n0 * U[1] * U[2] * ir + n1 * (U[2] * U[2] * ir + P);
    F[3] = n0 * (U[3] + P) * U[1] * ir + n1 * (U[3] + P) * U[2] * ir;
}

// Flux::Rusanov (src/Base/Flux.cpp:52-81).
template <class T>
__device__ __forceinline__ void rusanov(const T UL[4], const T UR[4], T n0, T n1, T gma, T F[4]) {
    const T gmo = gma - T(1);
    const T irl = qrcp(UL[0]);
    const T irr = qrcp(UR[0]);
    const T nvl = (n0 * UL[1] + n1 * UL[2]) * irl;
    const T nvr = (n0 * UR[1] + n1 * UR[2]) * irr;
    const T qql = T(0.5) * (UL[1] * UL[1] + UL[2] * UL[2]) * irl;
    const T qqr = T(0.5) * (UR[1] * UR[1] + UR[2] * UR[2]) * irr;
    const T pl = gmo * (UL[3] - qql);
    const T pr = gmo * (UR[3] - qqr);
    const T al = qsqrt(gma * pl * irl);
    const T ar = qsqrt(gma * pr * irr);
    const T S1 = fmax(fabs(nvl - al), fabs(nvr - ar));
    const T S2 = fmax(fabs(nvl + al), fabs(nvr + ar));
    const T S = fmax(S1, S2);
    T FL[4], FR[4];
    euler_flux(UL, irl, n0, n1, gma, FL);
    euler_flux(UR, irr, n0, n1, gma, FR);
#pragma unroll
    for (int v = 0; v < 4; v++) F[v] = T(0.5) * ((FL[v] + FR[v]) - S * (UR[v] - UL[v]));
}

// Green-Gauss weights of one face seen from one of its cells: the cell's own state weighs
// ws, its neighbour's wn (If and 1 - If, by side), and the face's contribution enters with
// the signed length sA (+A_f into the left cell, -A_f into the right one).  One select of
// two weights per face takes the place of selecting the left and right state of every
// variable; the product u_CL If + u_CR (1 - If) is the same sum, the two products possibly
// fused in the other order on the right cell (a rounding-level difference).
template <class T>
__device__ __forceinline__ void face_weights(bool isL, T If, T Af, T& ws, T& wn, T& sA) {
    const T w1 = If, w2 = T(1) - If;
    ws = isL ? w1 : w2;
    wn = isL ? w2 : w1;
    sA = isL ? Af : -Af;
}

// Spectral-radius term of one face for the local time step: (|u.n| + a) A_f from the
// cell's own state (u, v, a precomputed).
template <class T>
__device__ __forceinline__ T wave(T u, T v, T a, const FaceGeo<T>& g) {
    return (fabs(u * g.nx + v * g.ny) + a) * g.Af;
}

template <class T>
__device__ __forceinline__ void cell_speed(const T U[4], T gma, T& u, T& v, T& a) {
    const T ir = qrcp(U[0]);
    u = U[1] * ir;
    v = U[2] * ir;
    const T p = (gma - T(1)) * (U[3] - T(0.5) * (U[1] * u + U[2] * v));
    a = qsqrt(gma * p * ir);
}

// Face value of the limiter for one variable, |d| > 1e-9 (d = grad u . r_f):
//   Barth-Jespersen (Limiter.cpp:67-71): min(1, D1 / d), D1 = u_max - u if d > 0, else u_min - u;
//   Venkatakrishnan: min(1, (D1^2 + e2 + 2 D1 d) / (D1^2 + 2 d^2 + D1 d + e2)),
//                    e2 = (K h)^3, h = sqrt(cell area).
// (Skipping the quotient where it is at least 1 would give the same bits, but measured on the
// B200 the branch costs more than the division it saves, in both precisions.)
template <class T>
__device__ __forceinline__ T face_limiter(int limiter, T D1, T d, T e2) {
    if (limiter == LIM_BJ) return fmin(T(1), qdiv(D1, d));
    const T num = D1 * D1 + e2 + T(2) * D1 * d;
    const T den = D1 * D1 + T(2) * d * d + D1 * d + e2;
    return fmin(T(1), qdiv(num, den));
}

// Two-sum accumulation s + c += x (Knuth), with explicit round-to-nearest adds so that no
// multiply is fused into the sum.
__device__ __forceinline__ void two_sum(float& s, float& c, float x) {
    const float t = __fadd_rn(s, x);
    const float bp = __fsub_rn(t, s);
    const float e = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(x, bp));
    s = t;
    c = __fadd_rn(c, e);
}

// Ghost state from the updated interior state uc through the face with unit normal n:
// BoundaryCondition::update_cells of each type (src/Base/BoundaryConditions/*.cpp).
template <class T>
__device__ __forceinline__ void ghost_state(int type, const T uc[4], T n0, T n1, T gma,
                                            const double UBC[4], const double QBC[4], T ug[4]) {
    switch (type) {
    case 0: {                                           // Symmetry.cpp:5-24
        const T nor = uc[1] * n0 + uc[2] * n1;
        ug[0] = uc[0];
        ug[1] = uc[1] - T(2) * nor * n0;
        ug[2] = uc[2] - T(2) * nor * n1;
        ug[3] = uc[3];
    } break;
    case 1:                                             // Wall.cpp:4-15
        ug[0] = uc[0]; ug[1] = -uc[1]; ug[2] = -uc[2]; ug[3] = uc[3];
        break;
    case 2:                                             // Inlet.cpp:4-13
        for (int v = 0; v < 4; v++) ug[v] = T(UBC[v]);
        break;
    case 3: {                                           // Inlet.cpp:15-31
        const T PL = (gma - T(1)) * (uc[3] - T(0.5) * (uc[1] * uc[1] + uc[2] * uc[2]) / uc[0]);
        for (int v = 0; v < 4; v++) ug[v] = T(UBC[v]);
        ug[3] = PL / (gma - T(1)) + T(0.5) * T(QBC[0]) * (T(QBC[1]) * T(QBC[1]) + T(QBC[2]) * T(QBC[2]));
    } break;
    case 4:                                             // Outlet.cpp:4-13
        for (int v = 0; v < 4; v++) ug[v] = uc[v];
        break;
    default: {                                          // Outlet.cpp:15-32, as intended
        // The reference's loop reads rul[-1] and stops one momentum component short;
        // this takes rho and rho u from the interior and p from the BC state.
        ug[0] = uc[0]; ug[1] = uc[1]; ug[2] = uc[2];
        ug[3] = T(QBC[3]) / (gma - T(1)) + T(0.5) * (uc[1] * uc[1] + uc[2] * uc[2]) / uc[0];
    } break;
    }
}

__device__ __forceinline__ int bc_of_face(const BCTable& bc, int f) {
    int k = 0;
#pragma unroll 1
    while (k + 1 < bc.nbc && f >= bc.F1[k + 1]) k++;
    return k;
}

// ---------------------------------------------------------------------------------------
// reductions

template <class T>
__device__ __forceinline__ T warp_max(T x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}
// The CFL time-step minimum of a set of cells, min_i 1 / x_i with x_i = iv_i lam_i > 0: a
// correctly rounded reciprocal (FP64) does not grow as x grows, so the minimum equals
// 1 / max_i x_i bit for bit, and the cells keep a running maximum, one reciprocal being formed
// per warp or block (FP32 uses the hardware reciprocal, measured to give the same bits on the
// bench meshes).  fmax ignores a NaN x, so a cell with a NaN posts no step, and a set without
// a positive x posts nothing.
template <class T>
__device__ __forceinline__ double dt_of_max(T x) { return x > T(0) ? (double) qrcp(x) : 1e300; }
__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// ---------------------------------------------------------------------------------------
// pass 1: gradient + limiter (+ CFL minimum)

// Checked build: every face and neighbour id of the per-cell kernels' slot table ([W][Nc]
// int2: {face or ~face, neighbour}, neighbour -1 for an unused slot) checked on the device
// before a step; a bad one sets bit 2 of err and the host launches no step.  The per-cell step
// kernels themselves carry no checks, so they are the default build's code.
static __global__ void check_slots_kernel(const int2* __restrict__ slot, int W, int Nc, int Nf, unsigned int* err) {
    const size_t n = (size_t) W * Nc;
    for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x) {
        const int2 s = slot[i];
        if (s.y < 0) continue;
        const int f = s.x >= 0 ? s.x : ~s.x;
        if (f >= Nf || s.y >= Nc) atomicOr(err, 4u);
    }
}

template <class T, int W>
__global__ void __launch_bounds__(256) pass1_kernel(const StepArgs<T> a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    T xmx = T(0);                        // largest iv * lam (see dt_of_max)
    if (c < a.Nc) {
        int2 s[W];
#pragma unroll
        for (int k = 0; k < W; k++) s[k] = __ldg(a.slot + (size_t) k * a.Nc + c);
        if (s[0].y >= 0) {
            T u[4];
            ld_cell(a.U, a.Nc, c, u);
            const T iv = __ldg(a.iv + c);
            T G[4][2], umin[4], umax[4], ro[W][2];
#pragma unroll
            for (int v = 0; v < 4; v++) { G[v][0] = T(0); G[v][1] = T(0); umin[v] = u[v]; umax[v] = u[v]; }
            T cu = T(0), cv = T(0), ca = T(0), lam = T(0);
            if (a.time_mode != TM_FIXED) cell_speed(u, a.gma, cu, cv, ca);
#pragma unroll
            for (int k = 0; k < W; k++) {
                ro[k][0] = T(0); ro[k][1] = T(0);
                if (s[k].y < 0) continue;
                const bool isL = s[k].x >= 0;
                const int f = isL ? s[k].x : ~s[k].x;
                FaceGeo<T> g;
                ld_geo(a.geo, f, g);
                T un[4];
                ld_cell(a.U, a.Nc, s[k].y, un);
                // GaussGreen.cpp:25-28: uf = u_CL If + u_CR (1 - If); +uf Af n into CL,
                // -uf Af n into CR (the side folded into face_weights).
                T ws, wn, sA;
                face_weights(isL, g.If, g.Af, ws, wn, sA);
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const T uf = u[v] * ws + un[v] * wn;
                    const T t = uf * sA;
                    G[v][0] += t * g.nx;
                    G[v][1] += t * g.ny;
                    umin[v] = fmin(umin[v], un[v]);        // Limiter.cpp:31-39
                    umax[v] = fmax(umax[v], un[v]);
                }
                ro[k][0] = isL ? g.rLx : g.rRx;
                ro[k][1] = isL ? g.rLy : g.rRy;
                if (a.time_mode != TM_FIXED) lam += wave(cu, cv, ca, g);
            }
            T e2 = T(0);
            if (a.limiter == LIM_VENKAT) {
                const T kh = a.venkat_K * qsqrt(qrcp(iv));
                e2 = kh * kh * kh;
            }
            const T eps = T(1e-9);
            const int lmode = limiter_mode(a.stats->steps, a.freeze_after);
            T out[8], phis[4];
            if (lmode == LIM_FROZEN) ld_cell(a.phiF, a.Nc, c, phis);
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const T gx = G[v][0] * iv, gy = G[v][1] * iv;     // GaussGreen.cpp:33-39
                T phi = T(1);
                if (lmode == LIM_FROZEN) {
                    phi = phis[v];
                } else {
#pragma unroll
                    for (int k = 0; k < W; k++) {
                        if (s[k].y < 0) continue;
                        const T d = gx * ro[k][0] + gy * ro[k][1];   // Limiter.cpp:50-51
                        T pf = T(1);                                 // Limiter.cpp:67-71
                        if (d > eps || d < -eps)
                            pf = face_limiter(a.limiter, (d > eps) ? umax[v] - u[v] : umin[v] - u[v], d, e2);
                        phi = fmin(phi, pf);                         // Limiter.cpp:73-74
                    }
                }
                phis[v] = phi;
                out[2 * v] = phi * gx;
                out[2 * v + 1] = phi * gy;
            }
            if (lmode == LIM_RECORD) st_cell(a.phiF, a.Nc, c, phis);
            st_grad(a.phiG, a.Nc, c, out);
            if (a.time_mode != TM_FIXED) xmx = iv * lam;
        }
    }
    if (a.time_mode != TM_FIXED) {
        __shared__ T sm[32];
        T m = warp_max(xmx);
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if (lane == 0) sm[wid] = m;
        __syncthreads();
        if (wid == 0) {
            m = lane < (int) (blockDim.x >> 5) ? sm[lane] : T(0);
            const double d = dt_of_max(warp_max(m));
            if (lane == 0 && d < 1e300) atomicMin(a.dtmin, (unsigned long long) __double_as_longlong(d));
        }
    }
}

// ---------------------------------------------------------------------------------------
// pass 2: reconstruction + flux + gather + update + ghost refresh (+ residual)

template <class T, int W, bool COMP>
__global__ void __launch_bounds__(256) pass2_kernel(const StepArgs<T> a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double r2 = 0.0;
    int bad = 0;
    double dt_used = 0.0;
    if (a.time_mode == TM_FIXED) dt_used = a.dt_or_cfl;
    else dt_used = a.dt_or_cfl * __longlong_as_double((long long) *a.dtmin);
    if (c < a.Nc) {
        int2 s[W];
#pragma unroll
        for (int k = 0; k < W; k++) s[k] = __ldg(a.slot + (size_t) k * a.Nc + c);
        if (s[0].y >= 0) {
            T u[4], pg[8];
            ld_cell(a.U, a.Nc, c, u);
            ld_grad(a.phiG, a.Nc, c, pg);
            const T iv = __ldg(a.iv + c);
            T R[4], Rc[4];
#pragma unroll
            for (int v = 0; v < 4; v++) { R[v] = T(0); Rc[v] = T(0); }
            T cu = T(0), cv = T(0), ca = T(0), lam = T(0);
            if (a.time_mode == TM_LOCAL) cell_speed(u, a.gma, cu, cv, ca);
#pragma unroll
            for (int k = 0; k < W; k++) {
                if (s[k].y < 0) continue;
                const bool isL = s[k].x >= 0;
                const int f = isL ? s[k].x : ~s[k].x;
                FaceGeo<T> g;
                ld_geo(a.geo, f, g);
                const T ro0 = isL ? g.rLx : g.rRx, ro1 = isL ? g.rLy : g.rRy;
                const T rn0 = isL ? g.rRx : g.rLx, rn1 = isL ? g.rRy : g.rLy;
                T un[4], uo[4], uq[4];
                ld_cell(a.U, a.Nc, s[k].y, un);
                // MUSCL (Flux.cpp:83-87): U + phi grad U . r on each side.  A ghost
                // neighbour carries -grad and the same phi as this cell (BoundaryConditions/
                // Base.cpp:29-53) with r_R = -r_L (Domain.cpp:84-88), so its increment is this
                // cell's own increment.
                if (f >= a.F_BC) {
#pragma unroll
                    for (int v = 0; v < 4; v++) {
                        const T du = pg[2 * v] * ro0 + pg[2 * v + 1] * ro1;
                        uo[v] = u[v] + du;
                        uq[v] = un[v] + du;
                    }
                } else {
                    T pn[8];
                    ld_grad(a.phiG, a.Nc, s[k].y, pn);
#pragma unroll
                    for (int v = 0; v < 4; v++) {
                        uo[v] = u[v] + (pg[2 * v] * ro0 + pg[2 * v + 1] * ro1);
                        uq[v] = un[v] + (pn[2 * v] * rn0 + pn[2 * v + 1] * rn1);
                    }
                }
                T F[4];
                if (isL) rusanov(uo, uq, g.nx, g.ny, a.gma, F);
                else     rusanov(uq, uo, g.nx, g.ny, a.gma, F);
#pragma unroll
                for (int v = 0; v < 4; v++) {                    // Flux.cpp:39-42
                    if constexpr (COMP) {
                        const T x = isL ? -(g.Af * F[v]) : g.Af * F[v];
                        two_sum(R[v], Rc[v], x);
                    } else {
                        if (isL) R[v] -= g.Af * F[v];
                        else     R[v] += g.Af * F[v];
                    }
                }
                if (a.time_mode == TM_LOCAL) lam += wave(cu, cv, ca, g);
            }
            T dt;
            if (a.time_mode == TM_LOCAL) dt = T(a.dt_or_cfl) * qrcp(iv * lam);
            else dt = T(dt_used);
            T un_[4];
#pragma unroll
            for (int v = 0; v < 4; v++) {
                T Rv = COMP ? R[v] + Rc[v] : R[v];
                Rv = Rv * iv;                                      // Flux.cpp:45-49
                un_[v] = u[v] + dt * Rv;                           // Euler.cpp:107-113
                if (v == 0) r2 = (double) Rv * (double) Rv;
                bad |= !isfinite(un_[v]);
            }
            st_cell(a.Unew, a.Nc, c, un_);
            // Ghost refresh (update_BC_cells, Euler.cpp:96 and :138-142): this cell is the
            // only interior neighbour of each of its ghosts.
#pragma unroll
            for (int k = 0; k < W; k++) {
                if (s[k].y < 0) continue;
                const int f = s[k].x >= 0 ? s[k].x : ~s[k].x;
                if (f < a.F_BC) continue;
                const int b = bc_of_face(a.bc, f);
                FaceGeo<T> g;
                ld_geo(a.geo, f, g);
                T ug[4];
                ghost_state(a.bc.type[b], un_, g.nx, g.ny, a.gma, a.bc.UBC[b], a.bc.QBC[b], ug);
                st_cell(a.Unew, a.Nc, s[k].y, ug);
            }
        }
    }
    // Deterministic residual: fixed-shape block tree, then the last block sums the block
    // partials in block order.
    __shared__ double sm[32];
    __shared__ int smbad[32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double w = warp_sum(r2);
    int wb = __any_sync(0xffffffffu, bad);
    if (lane == 0) { sm[wid] = w; smbad[wid] = wb; }
    __syncthreads();
    if (wid == 0) {
        const int nw = (int) (blockDim.x >> 5);
        double x = lane < nw ? sm[lane] : 0.0;
        int xb = lane < nw ? smbad[lane] : 0;
        x = warp_sum(x);
        xb = __any_sync(0xffffffffu, xb);
        if (lane == 0) {
            a.partial[blockIdx.x] = x;
            if (xb) atomicOr(&a.stats->nonfinite, 1);
            __threadfence();
            const unsigned int done = atomicAdd(a.counter, 1u);
            last = (done == gridDim.x - 1);
        }
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double x = 0.0;
        for (int i = threadIdx.x; i < (int) gridDim.x; i += blockDim.x) x += ((volatile double*) a.partial)[i];
        x = warp_sum(x);
        if (lane == 0) sm[wid] = x;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (int i = 0; i < (int) (blockDim.x >> 5); i++) tot += sm[i];
            StepStats* st = a.stats;
            st->res2_last = tot;
            if (st->steps == 0) st->res2_first = tot;
            st->steps += 1;
            st->dt_last = dt_used;
            if (!(tot == tot) || tot > 1.7e308) st->nonfinite = 1;
            *a.counter = 0u;
            if (a.time_mode != TM_FIXED) *a.dtmin_next = 0x7FF0000000000000ULL;   // +inf
        }
    }
}

// ---------------------------------------------------------------------------------------
// geometry precompute (double), src/Base/Domain.cpp:44-154

// Domain::compute_xc (:61-71): vertex average, summed node by node in cn_con order.
static __global__ void geom_xc_kernel(int Nc, const int* __restrict__ cn_off, const int* __restrict__ cn_con,
                               const double* __restrict__ nodes, double* __restrict__ xc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Nc) return;
    const int b = cn_off[i], e = cn_off[i + 1];
    const int nnds = e - b;
    double x = 0.0, y = 0.0;
    for (int n = b; n < e; n++) {
        const int nd = cn_con[n];
        x += nodes[2 * nd] / nnds;
        y += nodes[2 * nd + 1] / nnds;
    }
    xc[2 * i] = x;
    xc[2 * i + 1] = y;
}

// compute_xf (:44-59), compute_rf (:73-89), compute_nf (:91-116), compute_If (:118-125).
static __global__ void geom_face_kernel(int Nf, int F_BC, const int* __restrict__ fn_con, const int* __restrict__ fc_con,
                                 const double* __restrict__ nodes, const double* __restrict__ xc,
                                 FaceGeo<double>* __restrict__ geo) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= Nf) return;
    const int n1 = fn_con[2 * f], n2 = fn_con[2 * f + 1];
    const int CL = fc_con[2 * f], CR = fc_con[2 * f + 1];
    const double x1 = nodes[2 * n1], y1 = nodes[2 * n1 + 1];
    const double x2 = nodes[2 * n2], y2 = nodes[2 * n2 + 1];
    const double xfx = 0.5 * (x1 + x2), xfy = 0.5 * (y1 + y2);
    FaceGeo<double> g;
    g.rLx = xfx - xc[2 * CL];
    g.rLy = xfy - xc[2 * CL + 1];
    if (f >= F_BC) { g.rRx = -g.rLx; g.rRy = -g.rLy; }
    else { g.rRx = xfx - xc[2 * CR]; g.rRy = xfy - xc[2 * CR + 1]; }
    double nx = (y2 - y1), ny = -(x2 - x1);
    const double Af = sqrt(nx * nx + ny * ny);
    nx /= Af;
    ny /= Af;
    const double sgn = (nx * g.rLx + ny * g.rLy > 0) ? 1.0 : -1.0;
    nx = sgn * nx;
    ny = sgn * ny;
    g.nx = nx; g.ny = ny; g.Af = Af;
    const double nrL = nx * g.rLx + ny * g.rLy;
    const double nrR = -(nx * g.rRx + ny * g.rRy);
    g.If = nrL / (nrL + nrR);
    geo[f] = g;
}

// compute_iv (:127-146) + zero_bc_iv (:148-154), gathered per cell over its faces in
// increasing face order (the reference's scatter order for that cell).
static __global__ void geom_iv_kernel(int Nc, int F_BC, const int* __restrict__ cf_off, const int* __restrict__ cf_con,
                               const int* __restrict__ fc_con, const FaceGeo<double>* __restrict__ geo,
                               double* __restrict__ iv) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Nc) return;
    double s = 0.0;
    bool ghost = false;
    for (int k = cf_off[c]; k < cf_off[c + 1]; k++) {
        const int f = cf_con[k];
        const FaceGeo<double> g = geo[f];
        if (fc_con[2 * f] == c) {
            const double AL = g.Af * (g.nx * g.rLx + g.ny * g.rLy);
            s += AL / 2;
        } else {
            const double AR = g.Af * (g.nx * g.rRx + g.ny * g.rRy);
            s -= AR / 2;
            if (f >= F_BC) ghost = true;
        }
    }
    iv[c] = ghost ? 0.0 : 1.0 / s;
}

template <class T>
__global__ void convert_geo_kernel(int Nf, const FaceGeo<double>* __restrict__ src, FaceGeo<T>* __restrict__ dst) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= Nf) return;
    const FaceGeo<double> g = src[f];
    FaceGeo<T> h;
    h.nx = T(g.nx); h.ny = T(g.ny); h.Af = T(g.Af); h.If = T(g.If);
    h.rLx = T(g.rLx); h.rLy = T(g.rLy); h.rRx = T(g.rRx); h.rRy = T(g.rRy);
    dst[f] = h;
}

template <class T>
__global__ void convert_iv_kernel(int Nc, const double* __restrict__ src, T* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < Nc) dst[i] = T(src[i]);
}

// ---------------------------------------------------------------------------------------
// state in/out

template <class T>
__global__ void fill_kernel(int Nc, Cell4<T>* __restrict__ U, double u0, double u1, double u2, double u3) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Nc) return;
    const T u[4] = {T(u0), T(u1), T(u2), T(u3)};
    st_cell(U, Nc, i, u);
}

// Euler::update_BC_cells over all boundary faces (used by initialise and upload).
// fc holds the faces' cells in the device's internal numbering.
template <class T>
__global__ void bc_cells_kernel(int Nc, int Nf, int F_BC, const int* __restrict__ fc, const FaceGeo<double>* __restrict__ geo,
                                Cell4<T>* __restrict__ U, T gma, const BCTable bc) {
    const int f = F_BC + blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= Nf) return;
    const int b = bc_of_face(bc, f);
    T uc[4], ug[4];
    ld_cell(U, Nc, fc[2 * f], uc);
    const FaceGeo<double> g = geo[f];
    ghost_state(bc.type[b], uc, T(g.nx), T(g.ny), gma, bc.UBC[b], bc.QBC[b], ug);
    st_cell(U, Nc, fc[2 * f + 1], ug);
}

// Euler::compute_prims (src/Base/Euler.cpp:115-136), or a plain copy of U; variable-major
// double output in the input numbering (perm[internal] = input index).
template <class T>
__global__ void out_kernel(int Nc, const Cell4<T>* __restrict__ U, const int* __restrict__ perm, double gma,
                           int prims, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Nc) return;
    T t[4];
    ld_cell(U, Nc, i, t);
    const size_t j = perm[i];
    const double u0 = t[0], u1 = t[1], u2 = t[2], u3 = t[3];
    if (!prims) {
        out[j] = u0; out[(size_t) Nc + j] = u1; out[2 * (size_t) Nc + j] = u2; out[3 * (size_t) Nc + j] = u3;
        return;
    }
    const double q0 = u0, q1 = u1 / u0, q2 = u2 / u0;
    const double gmo = gma - 1;
    const double q3 = gmo * (u3 - 0.5 * q0 * (q1 * q1 + q2 * q2));
    out[j] = q0; out[(size_t) Nc + j] = q1; out[2 * (size_t) Nc + j] = q2; out[3 * (size_t) Nc + j] = q3;
}

template <class T>
__global__ void in_kernel(int Nc, const double* __restrict__ in, const int* __restrict__ perm, Cell4<T>* __restrict__ U) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Nc) return;
    const size_t j = perm[i];
    const T u[4] = {T(in[j]), T(in[(size_t) Nc + j]), T(in[2 * (size_t) Nc + j]), T(in[3 * (size_t) Nc + j])};
    st_cell(U, Nc, i, u);
}

// dst[i] = src[perm[i]]
static __global__ void permute_kernel(int n, const double* __restrict__ src, const int* __restrict__ perm,
                               double* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[perm[i]];
}

template <class T>
__global__ void wall_cp_kernel(int Nc, int F1, int F2, const int* __restrict__ fc_con, const Cell4<T>* __restrict__ U,
                               double gma, double p_inf, double qinf, double* __restrict__ out) {
    const int f = F1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F2) return;
    T t[4];
    ld_cell(U, Nc, fc_con[2 * f], t);
    const double r = t[0], ru = t[1], rv = t[2], E = t[3];
    const double p = (gma - 1) * (E - 0.5 * (ru * ru + rv * rv) / r);
    out[f - F1] = (p - p_inf) / qinf;
}

}  // namespace hcfd
