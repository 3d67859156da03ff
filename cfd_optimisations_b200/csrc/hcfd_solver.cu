// Solver handle of the B200 solver: device memory, the per-handle stream, launches of the
// step kernels and the C ABI of include/hcfd_gpu.h for one mesh.
//
// Device numbering.  Cells live on the device in an internal order: the Morton order of the
// cell centres by default (so that consecutive cells are neighbours in space, whatever the
// input numbering), or the input order with keep_numbering.  Faces keep their input
// numbers, and each cell's faces are visited in increasing face number, so the internal
// order changes where data sits, never the arithmetic.  State crosses the ABI in the input
// numbering.
#include "hcfd_internal.hpp"
#include "hcfd_kernels.cuh"
#include "hcfd_tile.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

using hcfd::fail;

namespace {

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(HCFD_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

template <class P>
int dalloc(P** p, size_t n) {
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**) p, n * sizeof(P));
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(e == cudaErrorMemoryAllocation ? HCFD_ENOMEM : HCFD_ECUDA,
                    std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    return HCFD_OK;
}

inline int nblk(long long n, int b) { return (int) ((n + b - 1) / b); }

// Primitive -> conservative, BoundaryCondition::init (src/Base/BoundaryConditions/Base.cpp:18-22).
void prim_to_cons(const double* q, double gma, double* u) {
    u[0] = q[0];
    for (int v = 1; v < 4; v++) u[v] = q[0] * q[v];
    u[3] = q[3] / (gma - 1) + 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2]);
}

}  // namespace

// One tile plan of the tiled kernels and its device arrays.  Pass 1 and pass 2 may run on
// different tilings of the same internal cell order (pass 2, which computes each face flux
// once per tile, gains from larger tiles than pass 1 does).
struct TiledPass {
    hcfd::TilePlan plan;
    void* d_tgeo = nullptr;              // face records [entries], T
    unsigned* d_tmeta = nullptr;         // pack_meta words [entries]
    int *d_foff = nullptr, *d_hoff = nullptr, *d_halo = nullptr;
    short* d_cslot = nullptr;
    int* d_efid = nullptr;               // set-up only
    int block = 0;                       // compute threads per CTA
    int rec = 8;                         // values per face record (7: pass 2 on a plan of its own)
};

struct hcfd_solver {
    int device = 0, nsm = 0;
    cudaStream_t stream = nullptr;
    hcfd_params prm{};
    int Nc = 0, Nf = 0, Nn = 0, Ncol = 0, NBC = 0, F_BC = 0, Nreal = 0, W = 0;
    std::vector<int> coloff, coltag;
    bool bcs_set = false, initialised = false;
    hcfd::BCTable bc{};
    // device buffers (cells in internal order)
    int* d_fc = nullptr;                 // fc_con in internal cell numbers [2 Nf]
    int* d_perm = nullptr;               // internal -> input cell number
    int2* d_slot = nullptr;              // per-cell kernels: [W][Nc]
    hcfd::FaceGeo<double>* d_geo64 = nullptr;   // [Nf], input face order
    void* d_geoT = nullptr;              // per-cell kernels in float: FaceGeo<float> [Nf]
    void* d_iv = nullptr;                // T [Nc]
    void* d_U[2] = {nullptr, nullptr};   // Cell4<T> [Nc]
    void* d_phiG = nullptr;              // Grad8<T> [Nc]
    void* d_phiF = nullptr;              // Cell4<T> [Nc]: frozen limiter values
    double* d_io = nullptr;              // 4 Nc doubles staging for upload/download
    double* d_cp = nullptr;              // Nf doubles for the wall Cp
    unsigned long long* d_dtmin = nullptr;   // [2]
    double* d_partial = nullptr;
    unsigned int* d_counter = nullptr;
    unsigned int* d_err = nullptr;
    hcfd::StepStats* d_stats = nullptr;
    // tiled kernels
    TiledPass tp[2];                     // pass 1; pass 2 when it has its own tiling
    bool split = false;                  // pass 2 uses tp[1]
    size_t smem1 = 0, smem2 = 0;
    int grid1 = 0, grid2 = 0;
    // tile queues (d_counter[1] for pass 1, d_counter[2] for pass 2): CTAs that finish
    // early take more tiles; without, every CTA takes every grid-th tile
    bool queue1 = true, queue2 = false;
    bool tiled = false;
    int cur = 0;                         // which of d_U holds the state
    int block = 256;
    int partial_len = 0;
    // profiling
    // asynchronous snapshots (hcfd_gpu_snapshot): staging buffer, copy stream, and the event
    // after which the staging buffer may be overwritten
    double* d_snap = nullptr;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t snap_free = nullptr;
    bool snap_used = false;
    // two steps captured as one CUDA graph (the ping-pong buffers and dt slots return to
    // their start), replayed while the time mode, dt/CFL value and buffer parity stay the same
    cudaGraphExec_t graph = nullptr;
    int g_mode = -1, g_cur = -1;
    double g_value = 0.0;
    bool prof = false;
    int prof_every = 1;                  // record every prof_every-th step
    long long prof_count = 0;
    std::vector<cudaEvent_t> ev1, ev2;   // start/stop pairs per launch
    double ms1 = 0, ms2 = 0;
    long long n1 = 0, n2 = 0;

    // bounded waits of the tiled kernels (hcfd_gpu_test_waits changes them for tests)
    unsigned wait_polls = 1u << 22;
    int wait_skip_tile = -1;

    bool fp32() const { return prm.precision == HCFD_FP32; }
};

namespace {

void free_all(hcfd_solver* s) {
    if (!s) return;
    if (s->device >= 0) cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto e : s->ev1) cudaEventDestroy(e);
    for (auto e : s->ev2) cudaEventDestroy(e);
    void* ptrs[] = {s->d_fc, s->d_perm, s->d_slot, s->d_geo64, s->d_geoT, s->d_iv, s->d_U[0], s->d_U[1],
                    s->d_phiG, s->d_phiF, s->d_io, s->d_cp, s->d_dtmin, s->d_partial, s->d_counter, s->d_err, s->d_stats};
    for (void* p : ptrs) if (p) cudaFree(p);
    for (TiledPass& P : s->tp) {
        void* q[] = {P.d_tgeo, P.d_tmeta, P.d_foff, P.d_hoff, P.d_halo, P.d_cslot, P.d_efid};
        for (void* p : q) if (p) cudaFree(p);
    }
    if (s->graph) cudaGraphExecDestroy(s->graph);
    if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
    if (s->d_snap) cudaFree(s->d_snap);
    if (s->snap_free) cudaEventDestroy(s->snap_free);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->stream) cudaStreamDestroy(s->stream);
}

template <class T>
hcfd::StepArgs<T> step_args(hcfd_solver* s, int time_mode, double dt_or_cfl) {
    hcfd::StepArgs<T> a;
    a.U = (const hcfd::Cell4<T>*) s->d_U[s->cur];
    a.Unew = (hcfd::Cell4<T>*) s->d_U[1 - s->cur];
    a.phiG = (hcfd::Grad8<T>*) s->d_phiG;
    a.geo = std::is_same<T, double>::value ? (const hcfd::FaceGeo<T>*) s->d_geo64 : (const hcfd::FaceGeo<T>*) s->d_geoT;
    a.slot = s->d_slot;
    a.iv = (const T*) s->d_iv;
    a.dtmin = s->d_dtmin + s->cur;
    a.dtmin_next = s->d_dtmin + (1 - s->cur);
    a.partial = s->d_partial;
    a.counter = s->d_counter;
    a.stats = s->d_stats;
    a.Nc = s->Nc;
    a.F_BC = s->F_BC;
    a.limiter = s->prm.limiter;
    a.time_mode = time_mode;
    a.gma = T(s->prm.gma);
    a.venkat_K = T(s->prm.venkat_K);
    a.dt_or_cfl = dt_or_cfl;
    a.bc = s->bc;
    a.phiF = (hcfd::Cell4<T>*) s->d_phiF;
    a.freeze_after = s->prm.freeze_limiter_after;
    return a;
}

template <class T>
hcfd::TileArgs<T> tile_args(hcfd_solver* s, int time_mode, double dt_or_cfl, const TiledPass& P, int pass) {
    hcfd::TileArgs<T> a;
    int* q1 = s->queue1 ? (int*) s->d_counter + 1 : nullptr;
    int* q2 = s->queue2 ? (int*) s->d_counter + 2 : nullptr;
    a.claim = pass == 1 ? q1 : q2;
    a.claim_reset = pass == 1 ? q2 : q1;
    a.s = step_args<T>(s, time_mode, dt_or_cfl);
    a.tgeo = (const T*) P.d_tgeo;
    a.rec = P.rec;
    a.tmeta = P.d_tmeta;
    a.foff = P.d_foff;
    a.hoff = P.d_hoff;
    a.halo = P.d_halo;
    a.cslot = P.d_cslot;
    a.ntiles = P.plan.ntiles;
    a.B = P.plan.B;
    a.Wp = P.plan.Wp;
    a.Hmax = P.plan.Hmax;
    a.Fmax = P.plan.Fmax;
    a.nentries = (long long) P.plan.efid.size();
    a.nhalo = (long long) P.plan.halo.size();
    a.ncap = (long long) P.plan.ntiles * P.plan.B;
    a.err = s->d_err;
    a.polls = s->wait_polls;
    a.skip_tile = s->wait_skip_tile;
    a.ps = s->Nc;
    a.tiles = nullptr;
    a.inst_dt = nullptr;
    a.inst_dtmin = nullptr;
    a.inst_bc = nullptr;
    a.tile_r2 = nullptr;
    a.tile_bad = nullptr;
    a.par = 0;
    return a;
}

struct Ev {
    cudaEvent_t a = nullptr, b = nullptr;
};

int prof_begin(hcfd_solver* s, bool rec, Ev& e) {
    if (!rec) return HCFD_OK;
    CK(cudaEventCreate(&e.a));
    CK(cudaEventCreate(&e.b));
    CK(cudaEventRecord(e.a, s->stream));
    return HCFD_OK;
}
int prof_end(hcfd_solver* s, bool rec, Ev& e, std::vector<cudaEvent_t>& into) {
    if (!rec) return HCFD_OK;
    CK(cudaEventRecord(e.b, s->stream));
    into.push_back(e.a);
    into.push_back(e.b);
    return HCFD_OK;
}

template <class T, int W>
int launch_step(hcfd_solver* s, int time_mode, double dt_or_cfl) {
    Ev e1, e2;
    int rc;
    const bool rec = s->prof && (s->prof_count++ % s->prof_every == 0);
    if (s->tiled) {
        const TiledPass& P2 = s->split ? s->tp[1] : s->tp[0];
        const hcfd::TileArgs<T> a1 = tile_args<T>(s, time_mode, dt_or_cfl, s->tp[0], 1);
        const hcfd::TileArgs<T> a2 = tile_args<T>(s, time_mode, dt_or_cfl, P2, 2);
        if ((rc = prof_begin(s, rec, e1))) return rc;
        hcfd::tile_pass1_kernel<T, W, false><<<s->grid1, s->tp[0].block + 32, s->smem1, s->stream>>>(a1);
        if ((rc = prof_end(s, rec, e1, s->ev1))) return rc;
        if ((rc = prof_begin(s, rec, e2))) return rc;
        hcfd::tile_pass2_kernel<T, W, std::is_same<T, float>::value, false><<<s->grid2, P2.block + 32, s->smem2, s->stream>>>(a2);
        if ((rc = prof_end(s, rec, e2, s->ev2))) return rc;
    } else {
        const int grid = nblk(s->Nc, s->block);
        hcfd::StepArgs<T> a = step_args<T>(s, time_mode, dt_or_cfl);
        if ((rc = prof_begin(s, rec, e1))) return rc;
        hcfd::pass1_kernel<T, W><<<grid, s->block, 0, s->stream>>>(a);
        if ((rc = prof_end(s, rec, e1, s->ev1))) return rc;
        if ((rc = prof_begin(s, rec, e2))) return rc;
        hcfd::pass2_kernel<T, W, std::is_same<T, float>::value><<<grid, s->block, 0, s->stream>>>(a);
        if ((rc = prof_end(s, rec, e2, s->ev2))) return rc;
    }
    CK(cudaGetLastError());
    s->cur = 1 - s->cur;
    return HCFD_OK;
}

template <class T>
int launch_step_w(hcfd_solver* s, int time_mode, double dt_or_cfl) {
    switch (s->W) {
    case 3: return launch_step<T, 3>(s, time_mode, dt_or_cfl);
    case 4: return launch_step<T, 4>(s, time_mode, dt_or_cfl);
    default: return launch_step<T, 8>(s, time_mode, dt_or_cfl);
    }
}

// Shared-memory opt-in and persistent grid size of the tiled kernels for one (T, W).
template <class T, int W>
int setup_tiled_w(hcfd_solver* s) {
    const hcfd::TilePlan& P = s->tp[0].plan;
    const TiledPass& T2 = s->split ? s->tp[1] : s->tp[0];
    const hcfd::TilePlan& Q = T2.plan;
    s->smem1 = hcfd::TileSmem<T>(P.B, P.Hmax, P.Fmax, W, P.Wp, false).total;
    s->smem2 = hcfd::TileSmem<T>(Q.B, Q.Hmax, Q.Fmax, W, Q.Wp, true).total;
    int maxsm = 0;
    CK(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device));
    if ((int) s->smem2 > maxsm || (int) s->smem1 > maxsm) return fail(HCFD_EINVAL, "tile does not fit in shared memory");
    CK(cudaFuncSetAttribute(hcfd::tile_pass1_kernel<T, W, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) s->smem1));
    CK(cudaFuncSetAttribute(hcfd::tile_pass2_kernel<T, W, std::is_same<T, float>::value, false>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int) s->smem2));
    int b1 = 0, b2 = 0;
    // blocks of the tiled kernels: `block` compute threads + one producer warp
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, hcfd::tile_pass1_kernel<T, W, false>, s->tp[0].block + 32,
                                                     s->smem1));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, hcfd::tile_pass2_kernel<T, W, std::is_same<T, float>::value, false>,
                                                     T2.block + 32, s->smem2));
    if (b1 < 1 || b2 < 1) return fail(HCFD_EINVAL, "tiled kernels cannot be resident");
    s->grid1 = std::min(P.ntiles, b1 * s->nsm);
    s->grid2 = std::min(Q.ntiles, b2 * s->nsm);
    return HCFD_OK;
}

template <class T>
int setup_tiled(hcfd_solver* s) {
    switch (s->W) {
    case 3: return setup_tiled_w<T, 3>(s);
    case 4: return setup_tiled_w<T, 4>(s);
    default: return setup_tiled_w<T, 8>(s);
    }
}

template <class T>
int refresh_ghosts(hcfd_solver* s) {
    const int nbf = s->Nf - s->F_BC;
    if (nbf > 0)
        hcfd::bc_cells_kernel<T><<<nblk(nbf, 256), 256, 0, s->stream>>>(
            s->Nc, s->Nf, s->F_BC, s->d_fc, s->d_geo64, (hcfd::Cell4<T>*) s->d_U[s->cur], T(s->prm.gma), s->bc);
    CK(cudaGetLastError());
    return HCFD_OK;
}

int check_handle(hcfd_solver* s) {
    if (!s) return fail(HCFD_EINVAL, "null solver handle");
    CK(cudaSetDevice(s->device));
    return HCFD_OK;
}

int read_stats(hcfd_solver* s, hcfd_step_stats* out) {
    hcfd::StepStats st;
    unsigned int err = 0;
    CK(cudaMemcpyAsync(&st, s->d_stats, sizeof(st), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(&err, s->d_err, sizeof(err), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (out) {
        out->dt = st.dt_last;
        out->res_l2 = s->Nreal > 0 ? std::sqrt(st.res2_last / s->Nreal) : 0.0;
        out->res_first = s->Nreal > 0 ? std::sqrt(st.res2_first / s->Nreal) : 0.0;
        out->steps = st.steps;
        out->nonfinite = st.nonfinite;
    }
    if (err & 4u) return fail(HCFD_EINVAL, "checked build: a tile index was out of range (corrupt tile plan)");
    if (err) return fail(HCFD_ETIMEOUT, "a bounded device wait gave up (tile staging did not complete)");
    return st.nonfinite ? fail(HCFD_ENONFINITE, "a step produced a NaN or Inf") : HCFD_OK;
}

}  // namespace

extern "C" {

int hcfd_gpu_create(const hcfd_mesh_view* mv, const hcfd_params* prm, hcfd_solver** out) {
    hcfd::clear_error();
    if (!mv || !out) return fail(HCFD_EINVAL, "gpu_create: null argument");
    *out = nullptr;
    int rc = hcfd::validate_view(*mv);
    if (rc != HCFD_OK) return rc;
    hcfd_params p{1.4, HCFD_LIMITER_BJ, 5.0, HCFD_FP64, 0, HCFD_KERNEL_TILED, 0, 0, 0, 0};
    if (prm) p = *prm;
    if (!(p.gma > 1.0) || (p.limiter != HCFD_LIMITER_BJ && p.limiter != HCFD_LIMITER_VENKAT) ||
        (p.precision != HCFD_FP64 && p.precision != HCFD_FP32) || p.block < 0 || p.block > 1024 || (p.block % 32) ||
        (p.kernel != HCFD_KERNEL_TILED && p.kernel != HCFD_KERNEL_CELL) || p.tile < 0 || p.tile > 512 || (p.tile % 32) ||
        (p.kernel == HCFD_KERNEL_TILED && p.block > 256) || p.freeze_limiter_after < 0 ||
        p.tile2 < 0 || p.tile2 > 512 || (p.tile2 % 32))
        return fail(HCFD_EINVAL, "gpu_create: bad parameters");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return fail(HCFD_ECUDA, "gpu_create: no CUDA device");

    auto s = std::make_unique<hcfd_solver>();
    CK(cudaGetDevice(&s->device));
    CK(cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, s->device));
    s->prm = p;
    s->block = p.block ? p.block : 256;
    s->Nc = mv->Nc; s->Nf = mv->Nf; s->Nn = mv->Nn; s->Ncol = mv->Ncol; s->NBC = mv->NBCcol;
    s->coloff.assign(mv->coloff, mv->coloff + mv->Ncol + 1);
    s->coltag.assign(mv->coltag, mv->coltag + mv->Ncol);
    s->F_BC = s->coloff[s->Ncol - s->NBC];
    if (s->NBC > hcfd::MAXBC) return fail(HCFD_EINVAL, "gpu_create: more than 16 boundary colours");
    const int Nc = s->Nc, Nf = s->Nf;

    // Host-side topology: cell->face table, ghosts, internal order.
    std::vector<int> cf_off, cf_con;
    hcfd::build_cf(Nc, Nf, mv->fc_con, cf_off, cf_con);
    std::vector<char> ghost(Nc, 0);
    for (int f = s->F_BC; f < Nf; f++) ghost[mv->fc_con[2 * f + 1]] = 1;
    int maxdeg = 0;
    for (int c = 0; c < Nc; c++) {
        if (ghost[c]) continue;
        s->Nreal++;
        maxdeg = std::max(maxdeg, cf_off[c + 1] - cf_off[c]);
    }
    if (maxdeg > 8) return fail(HCFD_EINVAL, "gpu_create: a cell has more than 8 faces");
    s->W = maxdeg <= 3 ? 3 : maxdeg <= 4 ? 4 : 8;
    std::vector<int> perm;
    if (p.keep_numbering) { perm.resize(Nc); for (int i = 0; i < Nc; i++) perm[i] = i; }
    else perm = hcfd::morton_order(*mv);
    std::vector<int> iperm(Nc);
    for (int i = 0; i < Nc; i++) iperm[perm[i]] = i;
    std::vector<int> fc_int(2 * (size_t) Nf);
    for (size_t k = 0; k < fc_int.size(); k++) fc_int[k] = iperm[mv->fc_con[k]];
    std::vector<int> bc_first;
    for (int col = s->Ncol - s->NBC; col < s->Ncol; col++) bc_first.push_back(s->coloff[col]);

    s->tiled = (p.kernel == HCFD_KERNEL_TILED);
    std::vector<int2> slot;
    if (s->tiled) {
        // Pass 1 on tiles of `tile` cells, pass 2 on tiles of `tile2`.  When neither is given:
        // FP64 224 and 192 cells, FP32 256 and 128 (pass 2's flux work per tile is heavy in
        // FP64, and fewer tile cuts pay; measured on the B200), falling back to smaller
        // tiles where a tiling does not fit shared memory (scattered cells, as with
        // keep_numbering on a shuffled mesh, have large halos).  When only `tile` is given,
        // both passes use it.  One compute thread per tile cell unless `block` says otherwise.
        const bool f64 = p.precision == HCFD_FP64;
        int maxsm = 0;
        CK(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device));
        auto need = [&](const hcfd::TilePlan& Q, bool pass2) {
            return f64 ? hcfd::TileSmem<double>(Q.B, Q.Hmax, Q.Fmax, s->W, Q.Wp, pass2).total
                       : hcfd::TileSmem<float>(Q.B, Q.Hmax, Q.Fmax, s->W, Q.Wp, pass2).total;
        };
        std::vector<int> c1 = p.tile ? std::vector<int>{p.tile} : std::vector<int>{f64 ? 224 : 256, 128, 64};
        std::vector<int> c2 = p.tile2 ? std::vector<int>{p.tile2}
                                      : p.tile ? std::vector<int>{p.tile} : std::vector<int>{f64 ? 192 : 128, 128, 64};
        bool ok = false;
        for (int t : c1) {
            rc = hcfd::build_tile_plan(*mv, cf_off, cf_con, ghost, perm, s->F_BC, bc_first, t, s->W, s->tp[0].plan);
            if (rc != HCFD_OK) return rc;
            if (need(s->tp[0].plan, false) <= (size_t) maxsm) { ok = true; break; }
        }
        if (!ok) return fail(HCFD_EINVAL, "tile does not fit in shared memory");
        const int tile1 = s->tp[0].plan.B;
        s->tp[0].block = p.block ? p.block : std::min(tile1, 256);
        ok = false;
        for (int t : c2) {
            if (t == tile1) {
                if (need(s->tp[0].plan, true) <= (size_t) maxsm) { s->split = false; ok = true; break; }
                continue;
            }
            rc = hcfd::build_tile_plan(*mv, cf_off, cf_con, ghost, perm, s->F_BC, bc_first, t, s->W, s->tp[1].plan,
                                       true);
            if (rc != HCFD_OK) return rc;
            if (need(s->tp[1].plan, true) <= (size_t) maxsm) {
                s->split = true;
                s->tp[1].block = p.block ? p.block : std::min(t, 256);
                ok = true;
                break;
            }
        }
        if (!ok) return fail(HCFD_EINVAL, "tile does not fit in shared memory");
        if (!s->split) s->tp[1] = TiledPass();
    } else {
        // Per-cell kernels: slot-major table {face or ~face, neighbour}, internal numbering.
        slot.assign((size_t) s->W * Nc, make_int2(-1, -1));
        for (int ci = 0; ci < Nc; ci++) {
            const int u = perm[ci];
            if (ghost[u]) continue;
            int k = 0;
            for (int j = cf_off[u]; j < cf_off[u + 1]; j++, k++) {
                const int f = cf_con[j];
                const int L = mv->fc_con[2 * f], R = mv->fc_con[2 * f + 1];
                slot[(size_t) k * Nc + ci] = (L == u) ? make_int2(f, iperm[R]) : make_int2(~f, iperm[L]);
            }
        }
    }

    CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    hcfd_solver* h = s.get();
    auto bail = [&](int code) { free_all(h); s.release(); delete h; return code; };
    const bool f32 = p.precision == HCFD_FP32;
    const size_t tsz = f32 ? sizeof(float) : sizeof(double);
    if (s->tiled) {
        rc = f32 ? setup_tiled<float>(h) : setup_tiled<double>(h);
        if (rc) return bail(rc);
        h->partial_len = std::max(h->grid1, h->grid2);
    } else {
        h->partial_len = nblk(Nc, h->block);
    }
    int* d_fn = nullptr; int* d_fcu = nullptr; int* d_cnoff = nullptr; int* d_cncon = nullptr;
    int* d_cfoff = nullptr; int* d_cfcon = nullptr;
    double* d_nodes = nullptr; double* d_xc = nullptr; double* d_ivu = nullptr;
    auto free_tmp = [&]() {
        cudaStreamSynchronize(h->stream);
        void* t[] = {d_fn, d_fcu, d_cnoff, d_cncon, d_cfoff, d_cfcon, d_nodes, d_xc, d_ivu, h->tp[0].d_efid, h->tp[1].d_efid};
        for (void* q : t) if (q) cudaFree(q);
        h->tp[0].d_efid = h->tp[1].d_efid = nullptr;
    };
    const int ncn = mv->cn_off[Nc];
    // iv is read one whole tile at a time by the tiled kernels: pad it to full tiles.
    size_t niv = Nc;
    for (const TiledPass& P : h->tp) niv = std::max(niv, (size_t) P.plan.ntiles * P.plan.B);
    if ((rc = dalloc(&h->d_fc, 2 * (size_t) Nf)) || (rc = dalloc(&h->d_perm, Nc)) ||
        (rc = dalloc(&h->d_geo64, Nf)) || (rc = dalloc((char**) &h->d_iv, tsz * niv)) ||
        (rc = dalloc((char**) &h->d_U[0], tsz * 4 * Nc)) || (rc = dalloc((char**) &h->d_U[1], tsz * 4 * Nc)) ||
        (rc = dalloc((char**) &h->d_phiG, tsz * 8 * Nc)) || (rc = dalloc(&h->d_io, 4 * (size_t) Nc)) ||
        (p.freeze_limiter_after > 0 && (rc = dalloc((char**) &h->d_phiF, tsz * 4 * Nc))) ||
        (rc = dalloc(&h->d_cp, Nf)) || (rc = dalloc(&h->d_dtmin, 2)) || (rc = dalloc(&h->d_partial, h->partial_len)) ||
        (rc = dalloc(&h->d_counter, 4)) || (rc = dalloc(&h->d_err, 1)) || (rc = dalloc(&h->d_stats, 1)) ||
        (rc = dalloc(&d_fn, 2 * (size_t) Nf)) || (rc = dalloc(&d_fcu, 2 * (size_t) Nf)) ||
        (rc = dalloc(&d_cnoff, Nc + 1)) || (rc = dalloc(&d_cncon, ncn)) || (rc = dalloc(&d_cfoff, Nc + 1)) ||
        (rc = dalloc(&d_cfcon, cf_con.size())) || (rc = dalloc(&d_nodes, 2 * (size_t) h->Nn)) ||
        (rc = dalloc(&d_xc, 2 * (size_t) Nc)) || (rc = dalloc(&d_ivu, Nc))) {
        free_tmp();
        return bail(rc);
    }
    if (h->tiled) {
        for (int k = 0; k < (h->split ? 2 : 1); k++) {
            TiledPass& P = h->tp[k];
            const size_t E = P.plan.efid.size();
            P.rec = k == 1 ? 7 : 8;     // pass 2's own plan leaves out If, which only pass 1 reads
            if ((rc = dalloc((char**) &P.d_tgeo, tsz * P.rec * E)) || (rc = dalloc(&P.d_tmeta, E)) ||
                (rc = dalloc(&P.d_foff, P.plan.foff.size())) || (rc = dalloc(&P.d_hoff, P.plan.hoff.size())) ||
                (rc = dalloc(&P.d_halo, P.plan.halo.size())) || (rc = dalloc(&P.d_cslot, P.plan.cslot.size())) ||
                (rc = dalloc(&P.d_efid, E))) {
                free_tmp();
                return bail(rc);
            }
        }
    } else {
        if ((rc = dalloc(&h->d_slot, slot.size())) || (f32 && (rc = dalloc((char**) &h->d_geoT, tsz * 8 * (size_t) Nf)))) {
            free_tmp();
            return bail(rc);
        }
    }
    cudaStream_t st = h->stream;
    auto up = [&](void* dst, const void* src, size_t bytes) {
        return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st) : cudaSuccess;
    };
    cudaError_t ce = cudaSuccess;
    if (ce == cudaSuccess) ce = up(h->d_fc, fc_int.data(), 8 * (size_t) Nf);
    if (ce == cudaSuccess) ce = up(h->d_perm, perm.data(), 4 * (size_t) Nc);
    if (ce == cudaSuccess) ce = up(d_fcu, mv->fc_con, 8 * (size_t) Nf);
    if (ce == cudaSuccess) ce = up(d_fn, mv->fn_con, 8 * (size_t) Nf);
    if (ce == cudaSuccess) ce = up(d_cnoff, mv->cn_off, 4 * (size_t) (Nc + 1));
    if (ce == cudaSuccess) ce = up(d_cncon, mv->cn_con, 4 * (size_t) ncn);
    if (ce == cudaSuccess) ce = up(d_cfoff, cf_off.data(), 4 * cf_off.size());
    if (ce == cudaSuccess) ce = up(d_cfcon, cf_con.data(), 4 * cf_con.size());
    if (ce == cudaSuccess) ce = up(d_nodes, mv->nodes, 16 * (size_t) h->Nn);
    if (h->tiled) {
        for (int k = 0; k < (h->split ? 2 : 1); k++) {
            TiledPass& T = h->tp[k];
            const hcfd::TilePlan& P = T.plan;
            const std::vector<unsigned> mw = hcfd::packed_meta(P);
            if (ce == cudaSuccess) ce = up(T.d_tmeta, mw.data(), 4 * mw.size());
            if (ce == cudaSuccess) ce = up(T.d_foff, P.foff.data(), 4 * P.foff.size());
            if (ce == cudaSuccess) ce = up(T.d_hoff, P.hoff.data(), 4 * P.hoff.size());
            if (ce == cudaSuccess) ce = up(T.d_halo, P.halo.data(), 4 * P.halo.size());
            if (ce == cudaSuccess) ce = up(T.d_cslot, P.cslot.data(), 2 * P.cslot.size());
            if (ce == cudaSuccess) ce = up(T.d_efid, P.efid.data(), 4 * P.efid.size());
        }
    } else {
        if (ce == cudaSuccess) ce = up(h->d_slot, slot.data(), sizeof(int2) * slot.size());
    }
    if (ce == cudaSuccess) {
        // Geometry in double, input numbering (src/Base/Domain.cpp:4-154).
        hcfd::geom_xc_kernel<<<nblk(Nc, 256), 256, 0, st>>>(Nc, d_cnoff, d_cncon, d_nodes, d_xc);
        hcfd::geom_face_kernel<<<nblk(Nf, 256), 256, 0, st>>>(Nf, h->F_BC, d_fn, d_fcu, d_nodes, d_xc, h->d_geo64);
        hcfd::geom_iv_kernel<<<nblk(Nc, 256), 256, 0, st>>>(Nc, h->F_BC, d_cfoff, d_cfcon, d_fcu, h->d_geo64, d_ivu);
        // iv to the internal numbering, then to T.
        ce = cudaMemsetAsync(h->d_iv, 0, tsz * niv, st);
        hcfd::permute_kernel<<<nblk(Nc, 256), 256, 0, st>>>(Nc, d_ivu, h->d_perm, d_xc);
        if (f32) hcfd::convert_iv_kernel<float><<<nblk(Nc, 256), 256, 0, st>>>(Nc, d_xc, (float*) h->d_iv);
        else ce = cudaMemcpyAsync(h->d_iv, d_xc, sizeof(double) * Nc, cudaMemcpyDeviceToDevice, st);
        for (int k = 0; h->tiled && k < (h->split ? 2 : 1); k++) {
            TiledPass& T = h->tp[k];
            const int nt = T.plan.ntiles;
            if (T.plan.efid.empty()) continue;
            if (f32) hcfd::gather_geo_kernel<float><<<nt, 128, 0, st>>>(nt, T.d_foff, T.d_efid, h->d_geo64, (float*) T.d_tgeo, T.rec);
            else hcfd::gather_geo_kernel<double><<<nt, 128, 0, st>>>(nt, T.d_foff, T.d_efid, h->d_geo64, (double*) T.d_tgeo, T.rec);
        }
        if (!h->tiled && f32)
            hcfd::convert_geo_kernel<float><<<nblk(Nf, 256), 256, 0, st>>>(Nf, h->d_geo64, (hcfd::FaceGeo<float>*) h->d_geoT);
        if (ce == cudaSuccess) ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) {
        const unsigned long long inf2[2] = {0x7FF0000000000000ULL, 0x7FF0000000000000ULL};
        ce = up(h->d_dtmin, inf2, sizeof(inf2));
    }
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->d_counter, 0, 4 * sizeof(unsigned int), st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->d_err, 0, sizeof(unsigned int), st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->d_stats, 0, sizeof(hcfd::StepStats), st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->d_phiG, 0, tsz * 8 * Nc, st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->d_U[0], 0, tsz * 4 * Nc, st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->d_U[1], 0, tsz * 4 * Nc, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    free_tmp();
    if (ce != cudaSuccess) return bail(fail(HCFD_ECUDA, std::string("gpu_create: ") + cudaGetErrorString(ce)));
    *out = s.release();
    return HCFD_OK;
}

int hcfd_gpu_gather_bcs(hcfd_solver* s, const int* bcmap, int nbcmap, const double* qbc) {
    hcfd::clear_error();
    int rc = check_handle(s);
    if (rc) return rc;
    if (!bcmap || !qbc || nbcmap <= 0) return fail(HCFD_EINVAL, "gather_bcs: bad argument");
    // Euler::gather_BCs (src/Base/Euler.cpp:42-60).
    hcfd::BCTable bc{};
    bc.nbc = s->NBC;
    const int fcolBC = s->Ncol - s->NBC;
    for (int fcol = fcolBC; fcol < s->Ncol; fcol++) {
        const int b = fcol - fcolBC;
        const int tag = s->coltag[fcol];
        if (tag < 0 || tag >= nbcmap) return fail(HCFD_EINVAL, "gather_bcs: colour tag outside the BC map");
        const int t = bcmap[tag];
        if (t < HCFD_SYMMETRY || t > HCFD_SUBOUTLET) return fail(HCFD_EINVAL, "gather_bcs: unknown BC type");
        bc.type[b] = t;
        bc.F1[b] = s->coloff[fcol];
        for (int v = 0; v < 4; v++) bc.QBC[b][v] = qbc[4 * b + v];
        prim_to_cons(bc.QBC[b], s->prm.gma, bc.UBC[b]);
    }
    bc.F1[s->NBC] = s->Nf;
    s->bc = bc;
    s->bcs_set = true;
    return HCFD_OK;
}

int hcfd_gpu_initialise(hcfd_solver* s, const double* qic) {
    hcfd::clear_error();
    int rc = check_handle(s);
    if (rc) return rc;
    if (!qic) return fail(HCFD_EINVAL, "initialise: null state");
    if (!s->bcs_set && s->NBC > 0) return fail(HCFD_EINVAL, "initialise: call gather_bcs first");
    // Euler::initialise (src/Base/Euler.cpp:62-77).
    double u[4];
    prim_to_cons(qic, s->prm.gma, u);
    s->cur = 0;
    if (s->fp32()) hcfd::fill_kernel<float><<<nblk(s->Nc, 256), 256, 0, s->stream>>>(s->Nc, (hcfd::Cell4<float>*) s->d_U[0], u[0], u[1], u[2], u[3]);
    else hcfd::fill_kernel<double><<<nblk(s->Nc, 256), 256, 0, s->stream>>>(s->Nc, (hcfd::Cell4<double>*) s->d_U[0], u[0], u[1], u[2], u[3]);
    CK(cudaGetLastError());
    rc = s->fp32() ? refresh_ghosts<float>(s) : refresh_ghosts<double>(s);
    if (rc) return rc;
    CK(cudaMemsetAsync(s->d_stats, 0, sizeof(hcfd::StepStats), s->stream));
    CK(cudaMemsetAsync(s->d_err, 0, sizeof(unsigned int), s->stream));
    CK(cudaMemsetAsync(s->d_counter, 0, 4 * sizeof(unsigned int), s->stream));   // ticket, tile queues
    const unsigned long long inf2[2] = {0x7FF0000000000000ULL, 0x7FF0000000000000ULL};
    CK(cudaMemcpyAsync(s->d_dtmin, inf2, sizeof(inf2), cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->initialised = true;
    return HCFD_OK;
}

int hcfd_gpu_step(hcfd_solver* s, int nsteps, int time_mode, double dt_or_cfl, hcfd_step_stats* stats) {
    hcfd::clear_error();
    int rc = check_handle(s);
    if (rc) return rc;
    if (!s->initialised) return fail(HCFD_EINVAL, "step: call initialise first");
    if (nsteps < 0 || time_mode < HCFD_FIXED_DT || time_mode > HCFD_LOCAL_CFL || !std::isfinite(dt_or_cfl) || dt_or_cfl < 0)
        return fail(HCFD_EINVAL, "step: bad argument");
    if constexpr (hcfd::kChecked) {
        // checked build: the per-cell kernels' slot table is checked on the device before
        // any step (the tiled kernels check their plan's indices as they read them)
        if (!s->tiled && nsteps > 0) {
            const long long n = (long long) s->W * s->Nc;
            hcfd::check_slots_kernel<<<(int) std::min<long long>((n + 255) / 256, 1184), 256, 0, s->stream>>>(
                s->d_slot, s->W, s->Nc, s->Nf, s->d_err);
            CK(cudaGetLastError());
            unsigned int err = 0;
            CK(cudaMemcpyAsync(&err, s->d_err, sizeof(err), cudaMemcpyDeviceToHost, s->stream));
            CK(cudaStreamSynchronize(s->stream));
            if (err & 4u) return fail(HCFD_EINVAL, "checked build: a face or neighbour id of the slot table is out of range");
        }
    }
    int n = nsteps;
    while (n > 0) {
        // pairs of steps without per-kernel events run as the graph; profiled steps run eagerly
        const bool rec = s->prof && (s->prof_count % s->prof_every == 0 || (s->prof_count + 1) % s->prof_every == 0);
        if (n >= 2 && !rec) {
            if (s->graph && (s->g_mode != time_mode || s->g_value != dt_or_cfl || s->g_cur != s->cur)) {
                cudaGraphExecDestroy(s->graph);
                s->graph = nullptr;
            }
            if (!s->graph) {
                const int cur0 = s->cur;
                const bool prof = s->prof;
                s->prof = false;                 // no events inside the graph
                cudaGraph_t g;
                CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
                for (int k = 0; k < 2 && rc == HCFD_OK; k++)
                    rc = s->fp32() ? launch_step_w<float>(s, time_mode, dt_or_cfl) : launch_step_w<double>(s, time_mode, dt_or_cfl);
                const cudaError_t e = cudaStreamEndCapture(s->stream, &g);
                s->prof = prof;
                if (rc) return rc;
                if (e != cudaSuccess) return fail(HCFD_ECUDA, std::string("step: capture: ") + cudaGetErrorString(e));
                const cudaError_t ei = cudaGraphInstantiate(&s->graph, g, 0);
                cudaGraphDestroy(g);
                if (ei != cudaSuccess) {
                    s->graph = nullptr;
                    return fail(HCFD_ECUDA, std::string("step: instantiate: ") + cudaGetErrorString(ei));
                }
                s->g_mode = time_mode;
                s->g_value = dt_or_cfl;
                s->g_cur = cur0;   // the capture flipped cur twice: back where it started
            }
            CK(cudaGraphLaunch(s->graph, s->stream));
            if (s->prof) s->prof_count += 2;
            n -= 2;
        } else {
            rc = s->fp32() ? launch_step_w<float>(s, time_mode, dt_or_cfl) : launch_step_w<double>(s, time_mode, dt_or_cfl);
            if (rc) return rc;
            n -= 1;
        }
    }
    if (stats) return read_stats(s, stats);
    return HCFD_OK;
}

int hcfd_gpu_test_waits(hcfd_solver* s, unsigned polls, int skip_tile) {
    hcfd::clear_error();
    int rc = check_handle(s);
    if (rc) return rc;
    if (polls > (1u << 30)) return fail(HCFD_EINVAL, "test_waits: poll limit above 2^30");
    s->wait_polls = polls ? polls : (1u << 22);
    s->wait_skip_tile = skip_tile < 0 ? -1 : skip_tile;
    if (s->graph) {                      // the kernel arguments live in the graph
        CK(cudaStreamSynchronize(s->stream));
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    return HCFD_OK;
}

int hcfd_gpu_stats(hcfd_solver* s, hcfd_step_stats* stats) {
    hcfd::clear_error();
    int rc = check_handle(s);
    if (rc) return rc;
    return read_stats(s, stats);
}

int hcfd_gpu_sync(hcfd_solver* s) {
    hcfd::clear_error();
    int rc = check_handle(s);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->stream));
    return read_stats(s, nullptr);
}

int hcfd_gpu_download(hcfd_solver* s, int prims, double* const* out) {
    hcfd::clear_error();
    int rc = check_handle(s);
    if (rc) return rc;
    if (!out) return fail(HCFD_EINVAL, "download: null output");
    for (int v = 0; v < 4; v++) if (!out[v]) return fail(HCFD_EINVAL, "download: null output array");
    if (s->fp32()) hcfd::out_kernel<float><<<nblk(s->Nc, 256), 256, 0, s->stream>>>(s->Nc, (const hcfd::Cell4<float>*) s->d_U[s->cur], s->d_perm, s->prm.gma, prims, s->d_io);
    else hcfd::out_kernel<double><<<nblk(s->Nc, 256), 256, 0, s->stream>>>(s->Nc, (const hcfd::Cell4<double>*) s->d_U[s->cur], s->d_perm, s->prm.gma, prims, s->d_io);
    CK(cudaGetLastError());
    for (int v = 0; v < 4; v++)
        CK(cudaMemcpyAsync(out[v], s->d_io + (size_t) v * s->Nc, sizeof(double) * s->Nc, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return HCFD_OK;
}

int hcfd_gpu_upload(hcfd_solver* s, const double* const* in) {
    hcfd::clear_error();
    int rc = check_handle(s);
    if (rc) return rc;
    if (!in) return fail(HCFD_EINVAL, "upload: null input");
    for (int v = 0; v < 4; v++) {
        if (!in[v]) return fail(HCFD_EINVAL, "upload: null input array");
        CK(cudaMemcpyAsync(s->d_io + (size_t) v * s->Nc, in[v], sizeof(double) * s->Nc, cudaMemcpyHostToDevice, s->stream));
    }
    if (s->fp32()) hcfd::in_kernel<float><<<nblk(s->Nc, 256), 256, 0, s->stream>>>(s->Nc, s->d_io, s->d_perm, (hcfd::Cell4<float>*) s->d_U[s->cur]);
    else hcfd::in_kernel<double><<<nblk(s->Nc, 256), 256, 0, s->stream>>>(s->Nc, s->d_io, s->d_perm, (hcfd::Cell4<double>*) s->d_U[s->cur]);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    s->initialised = true;
    return HCFD_OK;
}

}  // extern "C"

// A snapshot in flight: done when its copies to the host have landed.
struct hcfd_snapshot {
    cudaEvent_t done = nullptr;
    int device = 0;
};

extern "C" {

int hcfd_gpu_snapshot(hcfd_solver* s, int prims, double* const* host, hcfd_snapshot** ticket) {
    hcfd::clear_error();
    int rc = check_handle(s);
    if (rc) return rc;
    if (!host || !ticket) return fail(HCFD_EINVAL, "snapshot: null argument");
    for (int v = 0; v < 4; v++) if (!host[v]) return fail(HCFD_EINVAL, "snapshot: null host array");
    *ticket = nullptr;
    if (!s->d_snap) {
        // first snapshot: staging buffer, copy stream and event (allocates once)
        CK(cudaMalloc((void**) &s->d_snap, sizeof(double) * 4 * (size_t) s->Nc));
        CK(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&s->snap_free, cudaEventDisableTiming));
    }
    auto t = std::make_unique<hcfd_snapshot>();
    t->device = s->device;
    CK(cudaEventCreateWithFlags(&t->done, cudaEventDisableTiming));
    auto bail = [&](int code) { cudaEventDestroy(t->done); return code; };
    cudaError_t e = cudaSuccess;
    // the staging buffer is free once the previous snapshot's copies have landed
    if (s->snap_used) e = cudaStreamWaitEvent(s->stream, s->snap_free, 0);
    if (e == cudaSuccess) {
        if (s->fp32()) hcfd::out_kernel<float><<<nblk(s->Nc, 256), 256, 0, s->stream>>>(s->Nc, (const hcfd::Cell4<float>*) s->d_U[s->cur], s->d_perm, s->prm.gma, prims, s->d_snap);
        else hcfd::out_kernel<double><<<nblk(s->Nc, 256), 256, 0, s->stream>>>(s->Nc, (const hcfd::Cell4<double>*) s->d_U[s->cur], s->d_perm, s->prm.gma, prims, s->d_snap);
        e = cudaGetLastError();
    }
    // the copy stream starts when the conversion is done; the solver stream goes on stepping
    cudaEvent_t ready = nullptr;
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ready, s->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s->copy_stream, ready, 0);
    if (ready) cudaEventDestroy(ready);
    for (int v = 0; v < 4 && e == cudaSuccess; v++)
        e = cudaMemcpyAsync(host[v], s->d_snap + (size_t) v * s->Nc, sizeof(double) * s->Nc, cudaMemcpyDeviceToHost,
                            s->copy_stream);
    if (e == cudaSuccess) e = cudaEventRecord(s->snap_free, s->copy_stream);
    if (e == cudaSuccess) e = cudaEventRecord(t->done, s->copy_stream);
    if (e != cudaSuccess) return bail(fail(HCFD_ECUDA, std::string("snapshot: ") + cudaGetErrorString(e)));
    s->snap_used = true;
    *ticket = t.release();
    return HCFD_OK;
}

int hcfd_snapshot_wait(hcfd_snapshot* t) {
    hcfd::clear_error();
    if (!t) return fail(HCFD_EINVAL, "snapshot_wait: null ticket");
    const cudaError_t e = cudaEventSynchronize(t->done);
    if (e != cudaSuccess) return fail(HCFD_ECUDA, std::string("snapshot_wait: ") + cudaGetErrorString(e));
    return HCFD_OK;
}

void hcfd_snapshot_free(hcfd_snapshot* t) {
    if (!t) return;
    if (t->done) {
        cudaEventSynchronize(t->done);
        cudaEventDestroy(t->done);
    }
    delete t;
}

// Exact snapshot of a solve: the conservative state (all cells, input numbering), the step
// statistics and, with limiter freezing, the recorded limiter values.
int hcfd_gpu_checkpoint(hcfd_solver* s, const char* path) {
    hcfd::clear_error();
    int rc = check_handle(s);
    if (rc) return rc;
    if (!path) return fail(HCFD_EINVAL, "checkpoint: null path");
    if (!s->initialised) return fail(HCFD_EINVAL, "checkpoint: solver not initialised");
    const size_t n = 4 * (size_t) s->Nc;
    std::vector<double> U(n), phi;
    hcfd::StepStats st{};
    auto grab = [&](const void* src, std::vector<double>& dst) -> int {
        if (s->fp32()) hcfd::out_kernel<float><<<nblk(s->Nc, 256), 256, 0, s->stream>>>(s->Nc, (const hcfd::Cell4<float>*) src, s->d_perm, s->prm.gma, 0, s->d_io);
        else hcfd::out_kernel<double><<<nblk(s->Nc, 256), 256, 0, s->stream>>>(s->Nc, (const hcfd::Cell4<double>*) src, s->d_perm, s->prm.gma, 0, s->d_io);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(dst.data(), s->d_io, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        return HCFD_OK;
    };
    if ((rc = grab(s->d_U[s->cur], U))) return rc;
    if (s->d_phiF) {
        phi.resize(n);
        if ((rc = grab(s->d_phiF, phi))) return rc;
    }
    CK(cudaMemcpyAsync(&st, s->d_stats, sizeof(st), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    hcfd::CkptHeader h{};
    std::memcpy(h.magic, "HCFDCKP1", 8);
    h.version = 1;
    h.precision = s->prm.precision;
    h.Nc = s->Nc;
    h.has_phiF = s->d_phiF ? 1 : 0;
    h.steps = st.steps;
    h.res2_first = st.res2_first;
    h.res2_last = st.res2_last;
    h.dt_last = st.dt_last;
    h.nonfinite = st.nonfinite;
    return hcfd::ckpt_write(path, h, U, s->d_phiF ? &phi : nullptr);
}

int hcfd_gpu_restore(hcfd_solver* s, const char* path) {
    hcfd::clear_error();
    int rc = check_handle(s);
    if (rc) return rc;
    if (!path) return fail(HCFD_EINVAL, "restore: null path");
    hcfd::CkptHeader h;
    std::vector<double> U, phi;
    if ((rc = hcfd::ckpt_read(path, h, &U, &phi))) return rc;
    if (h.Nc != s->Nc) return fail(HCFD_EINVAL, "restore: the checkpoint is of a mesh with another cell count");
    if (h.precision != s->prm.precision) return fail(HCFD_EINVAL, "restore: the checkpoint is of another precision");
    if ((h.has_phiF != 0) != (s->d_phiF != nullptr))
        return fail(HCFD_EINVAL, "restore: limiter freezing differs between the checkpoint and this solver");
    auto put = [&](const std::vector<double>& src, void* dst) -> int {
        CK(cudaMemcpyAsync(s->d_io, src.data(), sizeof(double) * src.size(), cudaMemcpyHostToDevice, s->stream));
        if (s->fp32()) hcfd::in_kernel<float><<<nblk(s->Nc, 256), 256, 0, s->stream>>>(s->Nc, s->d_io, s->d_perm, (hcfd::Cell4<float>*) dst);
        else hcfd::in_kernel<double><<<nblk(s->Nc, 256), 256, 0, s->stream>>>(s->Nc, s->d_io, s->d_perm, (hcfd::Cell4<double>*) dst);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s->stream));   // d_io is reused by the next put
        return HCFD_OK;
    };
    if ((rc = put(U, s->d_U[s->cur]))) return rc;
    if (s->d_phiF && (rc = put(phi, s->d_phiF))) return rc;
    hcfd::StepStats st{};
    st.res2_first = h.res2_first;
    st.res2_last = h.res2_last;
    st.dt_last = h.dt_last;
    st.steps = h.steps;
    st.nonfinite = h.nonfinite;
    CK(cudaMemcpyAsync(s->d_stats, &st, sizeof(st), cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->initialised = true;
    return HCFD_OK;
}

int hcfd_gpu_wall_cp(hcfd_solver* s, int colour, double rho_inf, double p_inf, double speed_inf, double* out, int* n) {
    hcfd::clear_error();
    int rc = check_handle(s);
    if (rc) return rc;
    if (colour < 0 || colour >= s->Ncol || !out || !n) return fail(HCFD_EINVAL, "wall_cp: bad argument");
    const int F1 = s->coloff[colour], F2 = s->coloff[colour + 1];
    const double qinf = 0.5 * rho_inf * speed_inf * speed_inf;
    *n = F2 - F1;
    if (F2 == F1) return HCFD_OK;
    if (s->fp32()) hcfd::wall_cp_kernel<float><<<nblk(F2 - F1, 256), 256, 0, s->stream>>>(s->Nc, F1, F2, s->d_fc, (const hcfd::Cell4<float>*) s->d_U[s->cur], s->prm.gma, p_inf, qinf, s->d_cp);
    else hcfd::wall_cp_kernel<double><<<nblk(F2 - F1, 256), 256, 0, s->stream>>>(s->Nc, F1, F2, s->d_fc, (const hcfd::Cell4<double>*) s->d_U[s->cur], s->prm.gma, p_inf, qinf, s->d_cp);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, s->d_cp, sizeof(double) * (F2 - F1), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return HCFD_OK;
}

int hcfd_gpu_info(hcfd_solver* s, int* Nc, int* Nf, int* Nreal, int* slots) {
    if (!s) return fail(HCFD_EINVAL, "info: null handle");
    if (Nc) *Nc = s->Nc;
    if (Nf) *Nf = s->Nf;
    if (Nreal) *Nreal = s->Nreal;
    if (slots) *slots = s->W;
    return HCFD_OK;
}

int hcfd_gpu_profile(hcfd_solver* s, int enable) {
    int rc = check_handle(s);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->stream));
    for (auto e : s->ev1) cudaEventDestroy(e);
    for (auto e : s->ev2) cudaEventDestroy(e);
    s->ev1.clear(); s->ev2.clear();
    s->ms1 = s->ms2 = 0; s->n1 = s->n2 = 0;
    if (enable < 0) return fail(HCFD_EINVAL, "profile: negative sampling period");
    s->prof = enable != 0;
    s->prof_every = enable > 0 ? enable : 1;
    s->prof_count = 0;
    return HCFD_OK;
}

int hcfd_gpu_profile_read(hcfd_solver* s, double* ms_pass1, long long* n_pass1, double* ms_pass2, long long* n_pass2) {
    int rc = check_handle(s);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->stream));
    for (size_t i = 0; i + 1 < s->ev1.size(); i += 2) {
        float ms = 0; CK(cudaEventElapsedTime(&ms, s->ev1[i], s->ev1[i + 1])); s->ms1 += ms; s->n1++;
        cudaEventDestroy(s->ev1[i]); cudaEventDestroy(s->ev1[i + 1]);
    }
    for (size_t i = 0; i + 1 < s->ev2.size(); i += 2) {
        float ms = 0; CK(cudaEventElapsedTime(&ms, s->ev2[i], s->ev2[i + 1])); s->ms2 += ms; s->n2++;
        cudaEventDestroy(s->ev2[i]); cudaEventDestroy(s->ev2[i + 1]);
    }
    s->ev1.clear(); s->ev2.clear();
    if (ms_pass1) *ms_pass1 = s->ms1;
    if (n_pass1) *n_pass1 = s->n1;
    if (ms_pass2) *ms_pass2 = s->ms2;
    if (n_pass2) *n_pass2 = s->n2;
    return HCFD_OK;
}

int hcfd_gpu_step_timed(hcfd_solver* s, int nsteps, int time_mode, double dt_or_cfl, double* ms) {
    hcfd::clear_error();
    int rc = check_handle(s);
    if (rc) return rc;
    if (!ms) return fail(HCFD_EINVAL, "step_timed: null output");
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    CK(cudaEventRecord(a, s->stream));
    rc = hcfd_gpu_step(s, nsteps, time_mode, dt_or_cfl, nullptr);
    if (rc) { cudaEventDestroy(a); cudaEventDestroy(b); return rc; }
    CK(cudaEventRecord(b, s->stream));
    CK(cudaEventSynchronize(b));
    float t = 0;
    CK(cudaEventElapsedTime(&t, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms = t;
    return read_stats(s, nullptr);
}

int hcfd_gpu_launches_per_step(hcfd_solver* s) { return s ? 2 : 0; }

int hcfd_host_pin(void* p, size_t bytes) {
    hcfd::clear_error();
    if (!p || !bytes) return fail(HCFD_EINVAL, "host_pin: bad argument");
    CK(cudaHostRegister(p, bytes, cudaHostRegisterDefault));
    return HCFD_OK;
}

int hcfd_host_unpin(void* p) {
    hcfd::clear_error();
    if (!p) return fail(HCFD_EINVAL, "host_unpin: null pointer");
    CK(cudaHostUnregister(p));
    return HCFD_OK;
}

int hcfd_set_device(int device, int* count) {
    hcfd::clear_error();
    int n = 0;
    CK(cudaGetDeviceCount(&n));
    if (count) *count = n;
    if (device < 0 || device >= n) return fail(HCFD_EINVAL, "set_device: no such device");
    CK(cudaSetDevice(device));
    return HCFD_OK;
}

int hcfd_device_sync(void) {
    hcfd::clear_error();
    CK(cudaDeviceSynchronize());
    return HCFD_OK;
}

int hcfd_device_mem_info(size_t* free_bytes, size_t* total_bytes) {
    hcfd::clear_error();
    if (!free_bytes || !total_bytes) return fail(HCFD_EINVAL, "device_mem_info: null argument");
    CK(cudaMemGetInfo(free_bytes, total_bytes));
    return HCFD_OK;
}

void hcfd_gpu_destroy(hcfd_solver* s) {
    if (!s) return;
    free_all(s);
    delete s;
}

}  // extern "C"
