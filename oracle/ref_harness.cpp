// TEST INFRASTRUCTURE — not part of the product.
//
// Step-wise driver over the reference solver (Hasti-Jalal-Aldeen/CFD_Optimisations),
// compiled from the reference's own source files, unchanged, by oracle/Makefile into
// oracle/_ref/libhcfd_ref.so.  Only tests/, bench.py's CPU legs and smoke() load it, and
// only as the checker or as the timed CPU baseline.
//
// It calls the reference's phases in exactly the order of Euler::run's loop body
// (src/Base/Euler.cpp:86-96):
//     compute_gradient -> limit_gradient -> update_BC_grads -> update_BC_limiter
//     -> ComputeFlux -> add_residuals(dt) -> clear R -> update_BC_cells
// but takes dt per step (so a CFL-derived dt sequence can be replayed) and never touches
// the Writer (run() hard-codes "../sols/<Layout>", src/Base/Euler.cpp:22).
//
// The members it needs are private in the reference headers; the headers are included with
// `private` redefined to `public`, which changes access only, not layout.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <format>
#include <vector>
#include <thread>
#include <atomic>
#include <chrono>
#include <new>
#include <immintrin.h>

#define private public
#include "Global.hpp"
#include "Mesh.hpp"
#include "Writer.hpp"
#include "Base/Domain.hpp"
#include "Base/GradientSchemes.hpp"
#include "Base/Limiters.hpp"
#include "Base/Flux.hpp"
#include "Base/BoundaryConditions.hpp"
#include "Base/TimeIntegrators.hpp"
#include "SoA/Domain.hpp"
#include "SoA/GradientSchemes.hpp"
#include "SoA/Limiters.hpp"
#include "SoA/Flux.hpp"
#include "SoA/BoundaryConditions.hpp"
#include "SoA/TimeIntegrators.hpp"
#include "VEC/Domain.hpp"
#include "VEC/GradientSchemes.hpp"
#include "VEC/Limiters.hpp"
#include "VEC/Flux.hpp"
#include "VEC/BoundaryConditions.hpp"
#include "VEC/TimeIntegrators.hpp"
#include "AoSoA/Domain.hpp"
#include "AoSoA/GradientSchemes.hpp"
#include "AoSoA/Limiters.hpp"
#include "AoSoA/Flux.hpp"
#include "AoSoA/BoundaryConditions.hpp"
#include "AoSoA/TimeIntegrators.hpp"
#undef private

namespace {

// One reference solver instance of any layout whose state is `double* U[NVARS]`
// (Base, SoA, VEC, AoSoA).  CAoS and FAoS_CAoS are left out: their output differs from
// Base by ~4 % (phi indexed [var][cell] on a [cell][var] array,
// src/CAoS/BoundaryConditions/Base.cpp:49).
struct Instance {
    virtual ~Instance() {}
    virtual int Nc() const = 0;
    virtual void step(double dt) = 0;
    virtual void phase(int which, double dt) = 0;
    virtual double* U(int var) = 0;
    virtual double* Q(int var) = 0;
    virtual void prims() = 0;
    virtual double* G(int var) = 0;     // Base layout: G[var][dim*Nc + c]
    virtual double* phi(int var) = 0;
    virtual double* R(int var) = 0;
};

template <class Dom, class GG, class Lim, class Flx, class Eul, class BCT>
struct Layout final : Instance {
    Mesh* own_mesh;          // AoSoA rewrites the mesh it is given (src/AoSoA/Domain.cpp:69-92)
    Dom* d; GG* g; Lim* l; Flx* f; Eul* e;

    Layout(Mesh* mesh, Mesh* owned, double gma, const int* bcmap, int nbcmap,
           const double (*qbc)[NVARS], const double* qic) : own_mesh(owned) {
        d = new Dom(*mesh);
        g = new GG(*d);
        l = new Lim(*d);
        f = new Flx(NVARS, gma, *d);
        e = new Eul(NVARS, *d, *f, *g, *l);
        std::vector<BCT> map(nbcmap);
        for (int i = 0; i < nbcmap; i++) map[i] = (BCT) bcmap[i];
        e->gather_BCs(map.data(), qbc);
        e->initialise(qic);
    }
    ~Layout() override {
        delete e; delete f; delete l; delete g; delete d;
        delete own_mesh;
    }
    int Nc() const override { return d->Nc; }
    // src/Base/Euler.cpp:86-96, one loop iteration without the t bookkeeping.
    void step(double dt) override {
        e->grads.compute_gradient(e->nvars, e->U, e->G);
        e->limiter.limit_gradient(e->nvars, e->U, e->G, e->phi);
        e->update_BC_grads();
        e->update_BC_limiter();
        e->flux.ComputeFlux(e->U, e->G, e->phi, e->R);
        e->add_residuals(dt);
        for (int var = 0; var < e->nvars; var++) setarr(0, e->Nc, 0.0, e->R[var]);
        e->update_BC_cells();
    }
    void phase(int which, double dt) override {
        switch (which) {
        case 0: e->grads.compute_gradient(e->nvars, e->U, e->G); break;
        case 1: e->limiter.limit_gradient(e->nvars, e->U, e->G, e->phi); break;
        case 2: e->update_BC_grads(); e->update_BC_limiter(); break;
        case 3: e->flux.ComputeFlux(e->U, e->G, e->phi, e->R); break;
        case 4: e->add_residuals(dt); break;
        case 5: for (int var = 0; var < e->nvars; var++) setarr(0, e->Nc, 0.0, e->R[var]); break;
        case 6: e->update_BC_cells(); break;
        default: break;
        }
    }
    double* U(int v) override { return e->U[v]; }
    double* Q(int v) override { return e->Q[v]; }
    void prims() override { e->compute_prims(); }
    double* G(int v) override { return e->G[v]; }
    double* phi(int v) override { return e->phi[v]; }
    double* R(int v) override { return e->R[v]; }
};

using BaseL  = Layout<Base::Domain, Base::GaussGreen, Base::Limiter, Base::Flux, Base::Euler, Base::BCtype>;
using SoAL   = Layout<SoA::Domain, SoA::GaussGreen, SoA::Limiter, SoA::Flux, SoA::Euler, SoA::BCtype>;
using VECL   = Layout<VEC::Domain, VEC::GaussGreen, VEC::Limiter, VEC::Flux, VEC::Euler, VEC::BCtype>;
using AoSoAL = Layout<AoSoA::Domain, AoSoA::GaussGreen, AoSoA::Limiter, AoSoA::Flux, AoSoA::Euler, AoSoA::BCtype>;

bool file_ok(const char* path) {
    FILE* fp = fopen(path, "rb");
    if (!fp) return false;
    fclose(fp);
    return true;
}

Instance* make(const char* layout, Mesh* shared, const char* mesh_path, double gma,
               const int* bcmap, int nbcmap, const double* qbc, const double* qic) {
    auto q = reinterpret_cast<const double (*)[NVARS]>(qbc);
    std::string L(layout);
    if (L == "AoSoA") {
        Mesh* m = new Mesh(mesh_path);
        return new AoSoAL(m, m, gma, bcmap, nbcmap, q, qic);
    }
    Mesh* m = shared;
    Mesh* owned = nullptr;
    if (!m) { m = owned = new Mesh(mesh_path); }
    if (L == "Base") return new BaseL(m, owned, gma, bcmap, nbcmap, q, qic);
    if (L == "SoA")  return new SoAL(m, owned, gma, bcmap, nbcmap, q, qic);
    if (L == "VEC")  return new VECL(m, owned, gma, bcmap, nbcmap, q, qic);
    delete owned;
    return nullptr;
}

}  // namespace

extern "C" {

// Mesh header facts, read through the reference's own reader (src/Mesh.cpp:7-54).
int hcfd_ref_mesh_info(const char* path, int* out8) {
    if (!file_ok(path)) return -1;
    Mesh m(path);
    out8[0] = m.dim; out8[1] = m.Nn; out8[2] = m.Ncol; out8[3] = m.NBCcol;
    out8[4] = m.Nc;  out8[5] = m.Nf; out8[6] = m.N_pnames; out8[7] = m.cf_off[m.Nc];
    return 0;
}

// Copies the reference's CSR cell->face table (src/Mesh.cpp:88-117).
int hcfd_ref_mesh_cf(const char* path, int* cf_off, int* cf_con) {
    if (!file_ok(path)) return -1;
    Mesh m(path);
    std::memcpy(cf_off, m.cf_off, sizeof(int) * (m.Nc + 1));
    std::memcpy(cf_con, m.cf_con, sizeof(int) * m.cf_off[m.Nc]);
    return 0;
}

// Copies the Base geometry (src/Base/Domain.cpp:4-154) after zero_bc_iv, as Euler's
// constructor leaves it (src/Base/Euler.cpp:24).  Layout: rf[Nf*4], nf[Nf*2], Af[Nf],
// If[Nf], xc[Nc*2], iv[Nc].
int hcfd_ref_domain(const char* path, double* rf, double* nf, double* Af, double* If,
                    double* xc, double* iv) {
    if (!file_ok(path)) return -1;
    Mesh m(path);
    Base::Domain d(m);
    d.zero_bc_iv();
    std::memcpy(rf, d.rf, sizeof(double) * 4 * d.Nf);
    std::memcpy(nf, d.nf, sizeof(double) * 2 * d.Nf);
    std::memcpy(Af, d.Af, sizeof(double) * d.Nf);
    std::memcpy(If, d.If, sizeof(double) * d.Nf);
    std::memcpy(xc, d.xc, sizeof(double) * 2 * d.Nc);
    std::memcpy(iv, d.iv, sizeof(double) * d.Nc);
    return 0;
}

// layout: "Base", "SoA", "VEC" or "AoSoA".  bcmap is indexed by colour tag and qbc by BC
// index, as in Euler::gather_BCs (src/Base/Euler.cpp:42-60).  Returns NULL on failure.
void* hcfd_ref_create(const char* layout, const char* mesh_path, double gma,
                      const int* bcmap, int nbcmap, const double* qbc, const double* qic) {
    if (!file_ok(mesh_path)) return nullptr;
    return make(layout, nullptr, mesh_path, gma, bcmap, nbcmap, qbc, qic);
}

void hcfd_ref_free(void* h) { delete static_cast<Instance*>(h); }

int hcfd_ref_nc(void* h) { return static_cast<Instance*>(h)->Nc(); }

// nsteps steps; dt[i] for step i when ndt == nsteps, else dt[0] for every step.
int hcfd_ref_steps(void* h, int nsteps, const double* dt, int ndt) {
    Instance* in = static_cast<Instance*>(h);
    for (int s = 0; s < nsteps; s++) in->step(ndt == nsteps ? dt[s] : dt[0]);
    return 0;
}

int hcfd_ref_phase(void* h, int which, double dt) {
    static_cast<Instance*>(h)->phase(which, dt);
    return 0;
}

// which: 0 = U (conservative), 1 = Q (primitive, after compute_prims), 2 = phi, 3 = R.
// out holds 4 x Nc doubles, variable-major.
int hcfd_ref_get(void* h, int which, double* out) {
    Instance* in = static_cast<Instance*>(h);
    const int Nc = in->Nc();
    if (which == 1) in->prims();
    for (int v = 0; v < NVARS; v++) {
        const double* src = which == 0 ? in->U(v) : which == 1 ? in->Q(v)
                          : which == 2 ? in->phi(v) : in->R(v);
        std::memcpy(out + (size_t) v * Nc, src, sizeof(double) * Nc);
    }
    return 0;
}

// Base layout gradients: out holds 4 x 2 x Nc doubles, [var][dim][cell].
int hcfd_ref_get_G(void* h, double* out) {
    Instance* in = static_cast<Instance*>(h);
    const int Nc = in->Nc();
    for (int v = 0; v < NVARS; v++)
        std::memcpy(out + (size_t) v * 2 * Nc, in->G(v), sizeof(double) * 2 * Nc);
    return 0;
}

// Overwrites the conservative state (4 x Nc, variable-major).
int hcfd_ref_set_U(void* h, const double* in_u) {
    Instance* in = static_cast<Instance*>(h);
    const int Nc = in->Nc();
    for (int v = 0; v < NVARS; v++)
        std::memcpy(in->U(v), in_u + (size_t) v * Nc, sizeof(double) * Nc);
    return 0;
}

// Throughput timing of the reference loop: `nthreads` independent instances of one layout
// over one mesh, each built by its own thread (first-touch placement), `nwarm` untimed
// steps, a barrier, then `nsteps` timed steps with fixed dt.  The reference is single
// threaded, so the threads are independent replicas.  Writes the wall time of the timed
// region (first thread start to last thread end) to *secs.  Returns 0, or -1 if the mesh
// cannot be read or an instance cannot be built.
int hcfd_ref_bench(const char* layout, const char* mesh_path, double gma,
                   const int* bcmap, int nbcmap, const double* qbc, const double* qic,
                   int nthreads, int nwarm, int nsteps, double dt, double* secs) {
    if (!file_ok(mesh_path) || nthreads < 1) return -1;
    std::string L(layout);
    Mesh* shared = (L == "AoSoA") ? nullptr : new Mesh(mesh_path);
    std::atomic<int> ready{0}, failed{0};
    std::atomic<bool> go{false};
    std::vector<double> t_end(nthreads, 0.0);
    using clk = std::chrono::steady_clock;
    clk::time_point t0;
    std::vector<std::thread> th;
    for (int i = 0; i < nthreads; i++) {
        th.emplace_back([&, i]() {
            Instance* in = nullptr;
            try {
                in = make(layout, shared, mesh_path, gma, bcmap, nbcmap, qbc, qic);
            } catch (const std::bad_alloc&) { in = nullptr; }
            if (!in) failed++;
            else for (int s = 0; s < nwarm; s++) in->step(dt);
            ready++;
            while (!go.load()) std::this_thread::yield();
            if (in) {
                for (int s = 0; s < nsteps; s++) in->step(dt);
                t_end[i] = std::chrono::duration<double>(clk::now() - t0).count();
                delete in;
            }
        });
    }
    while (ready.load() < nthreads) std::this_thread::yield();
    t0 = clk::now();
    go = true;
    for (auto& t : th) t.join();
    delete shared;
    if (failed.load()) return -1;
    double mx = 0.0;
    for (double t : t_end) mx = t > mx ? t : mx;
    *secs = mx;
    return 0;
}

}  // extern "C"
