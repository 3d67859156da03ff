// hcfd_gpu.hpp — C++ drop-in for the reference's Base layout, running on the B200 solver.
//
// The classes below have the names, constructor signatures and methods of the reference's
// namespace Base (includes/Base/Domain.hpp, GradientSchemes.hpp, Limiters.hpp, Flux.hpp,
// BoundaryConditions.hpp, TimeIntegrators.hpp), so a driver written against the reference
// (src/Test.cpp:64-74) swaps `Base::` for `GPU::`.  Everything here is header-only and calls
// the C ABI of hcfd_gpu.h; link with -lhcfd_gpu.
//
// Differences from the reference, all deliberate:
//  - failures throw std::runtime_error with the library's message (the reference has no
//    error reporting at all);
//  - Euler writes its .hsln snapshots to `<prefix>_<k>.hsln` with prefix "../sols/GPU" by
//    default (the reference hard-codes "../sols/<Layout>", src/Base/Euler.cpp:22) and
//    creates nothing; set another prefix with set_output();
//  - Limiter takes an optional kind (Barth-Jespersen, as the reference, or
//    Venkatakrishnan) and Euler an optional time mode, precision and kernel choice;
//  - run() writes its snapshots without stopping the steps: each is copied to one of two
//    page-locked host buffers while the steps go on, and a writer thread writes the file
//    (the reference converts and writes between steps, src/Base/Euler.cpp:99-103); Q holds
//    the primitive state of the last step when run() returns.
#pragma once
#include "hcfd_gpu.h"

#include <algorithm>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace GPU {

inline void check(int rc) {
    if (rc != HCFD_OK) throw std::runtime_error(std::string("hcfd: ") + hcfd_last_error());
}

// includes/Base/BoundaryConditions.hpp:6-13
enum BCtype { SYMMETRY = HCFD_SYMMETRY, WALL = HCFD_WALL, SUPINLET = HCFD_SUPINLET,
              SUBINLET = HCFD_SUBINLET, SUPOUTLET = HCFD_SUPOUTLET, SUBOUTLET = HCFD_SUBOUTLET };

// Mesh(const char* fname) (includes/Mesh.hpp:15): the same public raw arrays, read by the
// library's checked .hmsh reader.
class Mesh {
public:
    int dim, Nn, Nc, Nf, Ncol, NBCcol, N_pnames;
    std::string* pnames;
    int *coltag, *coloff;
    double* nodes;
    int *fn_con, *fc_con;
    int *cf_con, *cf_off;
    int *cn_off, *cn_con;
    int *cc_off, *cc_con;

    explicit Mesh(const char* fname) {
        check(hcfd_mesh_load(fname, &m_));
        hcfd_mesh_view v;
        check(hcfd_mesh_view_of(m_, &v));
        dim = v.dim; Nn = v.Nn; Nc = v.Nc; Nf = v.Nf; Ncol = v.Ncol; NBCcol = v.NBCcol;
        coltag = const_cast<int*>(v.coltag); coloff = const_cast<int*>(v.coloff);
        nodes = const_cast<double*>(v.nodes);
        fn_con = const_cast<int*>(v.fn_con); fc_con = const_cast<int*>(v.fc_con);
        cn_off = const_cast<int*>(v.cn_off); cn_con = const_cast<int*>(v.cn_con);
        cc_off = const_cast<int*>(v.cc_off); cc_con = const_cast<int*>(v.cc_con);
        const int *o, *c;
        check(hcfd_mesh_cf(m_, &o, &c));
        cf_off = const_cast<int*>(o); cf_con = const_cast<int*>(c);
        for (N_pnames = 0; hcfd_mesh_pname(m_, N_pnames); N_pnames++) {}
        names_.resize(N_pnames);
        for (int k = 0; k < N_pnames; k++) names_[k] = hcfd_mesh_pname(m_, k);
        pnames = names_.data();
    }
    ~Mesh() { hcfd_mesh_free(m_); }
    Mesh(const Mesh&) = delete;
    Mesh& operator=(const Mesh&) = delete;

private:
    hcfd_mesh* m_ = nullptr;
    std::vector<std::string> names_;
};

// Domain(Mesh&) (includes/Base/Domain.hpp:26).  Accepts the reference's Mesh or GPU::Mesh
// (any type with the same public arrays); the geometry itself is computed on the device by
// the solver.
class Domain {
public:
    const int Nf, Nc;
    const int Ncol, NBC;
    hcfd_mesh_view view;
    std::vector<int> coltag;

    template <class MeshT>
    explicit Domain(MeshT& mesh)
        : Nf(mesh.Nf), Nc(mesh.Nc), Ncol(mesh.Ncol), NBC(mesh.NBCcol), coltag(mesh.coltag, mesh.coltag + mesh.Ncol) {
        view.dim = mesh.dim; view.Nn = mesh.Nn; view.Ncol = mesh.Ncol; view.NBCcol = mesh.NBCcol;
        view.Nc = mesh.Nc; view.Nf = mesh.Nf;
        view.coltag = mesh.coltag; view.coloff = mesh.coloff; view.nodes = mesh.nodes;
        view.fn_con = mesh.fn_con; view.fc_con = mesh.fc_con;
        view.cn_off = mesh.cn_off; view.cn_con = mesh.cn_con;
        view.cc_off = nullptr; view.cc_con = nullptr;
    }
};

// GradientScheme / GaussGreen (includes/Base/GradientSchemes.hpp:6-19): Green-Gauss is the
// gradient of the device step; these carry the domain.
class GradientScheme {
public:
    explicit GradientScheme(const Domain& domain) : Nc(domain.Nc), Nf(domain.Nf), domain(domain) {}
    virtual ~GradientScheme() {}
    const int Nc, Nf;
    const Domain& domain;
};
class GaussGreen : public GradientScheme {
public:
    using GradientScheme::GradientScheme;
};

// Limiter(const Domain&) (includes/Base/Limiters.hpp:8), Barth-Jespersen by default.
class Limiter {
public:
    explicit Limiter(const Domain& domain, int kind = HCFD_LIMITER_BJ, double K = 5.0)
        : kind(kind), K(K), domain(domain) {}
    const int kind;
    const double K;
    const Domain& domain;
};

// Flux(int nvars, double gma, const Domain&) (includes/Base/Flux.hpp:9): Rusanov.
class Flux {
public:
    Flux(int nvars, double gma, const Domain& domain) : nvars(nvars), gma(gma), domain(domain) {}
    const int nvars;
    const double gma;
    const Domain& domain;
};

// Euler(int nvars, Domain&, const Flux&, const GradientScheme&, Limiter&)
// (includes/Base/TimeIntegrators.hpp:11-45).
class Euler {
public:
    Euler(int nvars, Domain& domain, const Flux& flux, const GradientScheme& grads, Limiter& limiter,
          int precision = HCFD_FP64, int kernel = HCFD_KERNEL_TILED)
        : Nc(domain.Nc), Nf(domain.Nf), nvars(nvars), domain(domain), flux(flux) {
        (void) grads;
        if (nvars != 4) throw std::runtime_error("hcfd: nvars must be 4 (2-D Euler)");
        hcfd_params p{flux.gma, limiter.kind, limiter.K, precision, 0, kernel, 0, 0, 0};
        check(hcfd_gpu_create(&domain.view, &p, &solver_));
        for (int v = 0; v < 4; v++) {
            qbuf_[v].assign(Nc, 0.0);
            Q[v] = qbuf_[v].data();
        }
    }
    ~Euler() {
        if (writer_.joinable()) writer_.join();
        for (auto& b : snapbuf_) if (!b.empty()) hcfd_host_unpin(b.data());
        hcfd_gpu_destroy(solver_);
    }
    Euler(const Euler&) = delete;
    Euler& operator=(const Euler&) = delete;

    // src/Base/Euler.cpp:42-60
    void gather_BCs(const BCtype* BCmap, const double QBC[][4]) {
        const int nmap = *std::max_element(domain.coltag.begin(), domain.coltag.end()) + 1;
        std::vector<int> map(BCmap, BCmap + nmap);
        check(hcfd_gpu_gather_bcs(solver_, map.data(), nmap, &QBC[0][0]));
    }
    // src/Base/Euler.cpp:62-77
    void initialise(const double QIC[4]) { check(hcfd_gpu_initialise(solver_, QIC)); }
    // src/Base/Euler.cpp:79-105: fixed dt, a snapshot at t = 0 and each time t >= t_out.
    void run(double T, double dt, double dt_out) { run_mode(T, HCFD_FIXED_DT, dt, dt_out); }
    // The same loop with dt from a CFL number (global) instead of a fixed dt: runs until
    // t >= T, writing a snapshot each time t >= t_out.
    void run_cfl(double T, double cfl, double dt_out) { run_mode(T, HCFD_GLOBAL_CFL, cfl, dt_out); }
    // src/Base/Euler.cpp:115-136, into the host arrays Q.
    void compute_prims() { check(hcfd_gpu_download(solver_, 1, Q)); }
    void set_output(const std::string& prefix) { prefix_ = prefix; }
    hcfd_solver* handle() { return solver_; }

    double* Q[4];       // primitive variables of the last compute_prims, host memory
    const int Nc, Nf, nvars;

private:
    // Snapshot k goes to buffer k % 2 (its last user, writer k - 2, was joined at output
    // k - 1); the copy overlaps the wait for writer k - 1, then writer k takes over.
    void write_soln() {
        const int b = runcount_ % 2;
        if (snapbuf_[b].empty()) {
            snapbuf_[b].assign(4 * (size_t) Nc, 0.0);
            check(hcfd_host_pin(snapbuf_[b].data(), sizeof(double) * snapbuf_[b].size()));
        }
        double* arrs[4];
        for (int v = 0; v < 4; v++) arrs[v] = snapbuf_[b].data() + (size_t) v * Nc;
        hcfd_snapshot* t = nullptr;
        check(hcfd_gpu_snapshot(solver_, 1, arrs, &t));
        join_writer();
        const std::string fn = prefix_ + "_" + std::to_string(runcount_++) + ".hsln";
        const int nc = Nc;
        writer_ = std::thread([this, t, fn, b, nc]() {
            static const char* names[4] = {"Density", "Velocity_X", "Velocity_Y", "Pressure"};
            const double* out[4];
            for (int v = 0; v < 4; v++) out[v] = snapbuf_[b].data() + (size_t) v * nc;
            int rc = hcfd_snapshot_wait(t);
            if (rc == HCFD_OK) rc = hcfd_write_hsln(fn.c_str(), 4, names, nc, out);
            if (rc != HCFD_OK) writer_error_ = std::string("hcfd: ") + hcfd_last_error();
            hcfd_snapshot_free(t);
        });
    }
    void join_writer() {
        if (writer_.joinable()) writer_.join();
        if (!writer_error_.empty()) {
            const std::string e = writer_error_;
            writer_error_.clear();
            throw std::runtime_error(e);
        }
    }
    void run_mode(double T, int mode, double value, double dt_out) {
        double t = 0.0, t_out = dt_out;
        write_soln();
        if (mode == HCFD_FIXED_DT) {
            // the steps up to each output are counted with the reference's own t += dt
            while (t < T) {
                int n = 0;
                while (t < T) {
                    t += value;
                    n++;
                    if (t >= t_out) break;
                }
                check(hcfd_gpu_step(solver_, n, mode, value, nullptr));
                if (t >= t_out) {
                    write_soln();
                    t_out += dt_out;
                }
            }
        } else {
            while (t < T) {
                hcfd_step_stats st;
                check(hcfd_gpu_step(solver_, 1, mode, value, &st));
                t += st.dt;
                if (t >= t_out) {
                    write_soln();
                    t_out += dt_out;
                }
            }
        }
        join_writer();
        compute_prims();
    }

    Domain& domain;
    const Flux& flux;
    hcfd_solver* solver_ = nullptr;
    std::vector<double> qbuf_[4];
    std::string prefix_ = "../sols/GPU";
    int runcount_ = 0;
    std::vector<double> snapbuf_[2];      // page-locked snapshot buffers, 4 x Nc each
    std::thread writer_;
    std::string writer_error_;
};

}  // namespace GPU
