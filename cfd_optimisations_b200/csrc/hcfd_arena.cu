// Batched and served solves: many meshes packed into one flat device arena.
//
// The arena owns one set of device arrays sized from an HBM budget: cell planes (two
// state buffers, limited gradients, 1/area, slot tables), face-entry blocks (records and
// metadata) and halo lists.  Each admitted mesh (an instance) gets contiguous ranges in
// each (first-fit free lists on the host, so per-instance offsets), its own tile plan
// (hcfd_plan.cpp) with offsets added, its own BC table, dt or CFL number, dt minimum and
// statistics.  The tiled step kernels (hcfd_tile.cuh) run in arena mode over the list of
// all active tiles; a finalize kernel then forms each instance's residual from its tiles in
// tile order.  An instance's arithmetic is exactly that of the single-mesh solver with the
// same tile size, whatever else is in the arena, so a result is the same alone and in the
// mix.  A chunk of steps is captured once as a CUDA graph and replayed until the set of
// instances changes.
#include "hcfd_internal.hpp"
#include "hcfd_kernels.cuh"
#include "hcfd_tile.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

using hcfd::fail;
using hcfd::Cell4;

namespace {

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(HCFD_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

inline int nblk(long long n, int b) { return (int) ((n + b - 1) / b); }

// First-fit allocator over [0, capacity) with coalescing free list.
struct FreeList {
    std::map<size_t, size_t> free_;   // offset -> length
    size_t cap = 0, used = 0;
    void init(size_t capacity) { free_.clear(); cap = capacity; used = 0; if (cap) free_[0] = cap; }
    bool alloc(size_t n, size_t& off) {
        if (n == 0) { off = 0; return true; }
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                off = it->first;
                const size_t rest = it->second - n;
                free_.erase(it);
                if (rest) free_[off + n] = rest;
                used += n;
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t n) {
        if (n == 0) return;
        used -= n;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) { it->second += nx->second; free_.erase(nx); }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) { pv->second += it->second; free_.erase(it); }
        }
    }
};

struct Inst {
    bool active = false;
    int Nc = 0, Nf = 0, Nreal = 0, ntiles = 0, Hmax = 0, Fmax = 0;
    size_t c0 = 0, ncell = 0, e0 = 0, ne = 0, h0 = 0, nh = 0;
    int* d_perm = nullptr;                 // instance internal -> input cell number
    std::vector<int> tiles;                // 8 ints per tile, arena offsets
    double dt = 0;
    long long admitted_step = 0;
};

// Residual of each instance in two stages, both in an order fixed relative to the
// instance's first tile, so that it does not depend on where the instance sits in the arena.
// Stage 1: a block per chunk of kChunk per-warp partials of one instance (thread k takes
// partials k, k + 256, ..., then the threads in a fixed tree).
constexpr int kChunk = 8192;
__global__ void __launch_bounds__(256) arena_chunk_kernel(const int4* __restrict__ chunks,
                                                          const double* __restrict__ tile_r2,
                                                          const int* __restrict__ tile_bad, double* __restrict__ chunk_r2,
                                                          int* __restrict__ chunk_bad) {
    __shared__ double sx[8];
    __shared__ int sb[8];
    const int4 c = chunks[blockIdx.x];               // {act index, first partial, end, -}
    double x0 = 0.0, x1 = 0.0;
    int b = 0;
    int j = c.y + (int) threadIdx.x;
    for (; j + 256 < c.z; j += 512) {
        x0 += tile_r2[j];
        x1 += tile_r2[j + 256];
        b |= tile_bad[j] | tile_bad[j + 256];
    }
    for (; j < c.z; j += 256) { x0 += tile_r2[j]; b |= tile_bad[j]; }
    const double x = hcfd::warp_sum(x0 + x1);
    b = __any_sync(0xffffffffu, b);
    if ((threadIdx.x & 31) == 0) { sx[threadIdx.x >> 5] = x; sb[threadIdx.x >> 5] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        int bb = 0;
        for (int w = 0; w < 8; w++) { t += sx[w]; bb |= sb[w]; }
        chunk_r2[blockIdx.x] = t;
        chunk_bad[blockIdx.x] = bb;
    }
}

// Stage 2, per active instance {slot, first tile, end tile, first chunk}: its chunks in
// order, then the step statistics and dt bookkeeping.
__global__ void arena_finalize_kernel(int nact, int nchunks, const int4* __restrict__ act,
                                      const double* __restrict__ chunk_r2, const int* __restrict__ chunk_bad,
                                      const double* __restrict__ inst_dt, unsigned long long* inst_dtmin,
                                      hcfd::StepStats* stats, int time_mode, int par) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nact) return;
    const int4 d = act[i];
    const int slot = d.x, c0 = d.w, c1 = i + 1 < nact ? act[i + 1].w : nchunks;
    double x = 0.0;
    int b = 0;
    for (int c = c0; c < c1; c++) { x += chunk_r2[c]; b |= chunk_bad[c]; }
    hcfd::StepStats* st = stats + slot;
    st->res2_last = x;
    if (st->steps == 0) st->res2_first = x;
    st->steps += 1;
    const double v = inst_dt[slot];
    st->dt_last = time_mode == hcfd::TM_FIXED ? v : v * __longlong_as_double((long long) inst_dtmin[2 * slot + par]);
    if (b || !(x == x) || x > 1.7e308) st->nonfinite = 1;
    inst_dtmin[2 * slot + (1 - par)] = 0x7FF0000000000000ULL;
}

template <class T>
__global__ void arena_fill_kernel(size_t ps, size_t c0, int n, Cell4<T>* U, double u0, double u1, double u2, double u3) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const T u[4] = {T(u0), T(u1), T(u2), T(u3)};
    hcfd::st_cell(U, ps, (int) (c0 + i), u);
}

template <class T>
__global__ void arena_out_kernel(size_t ps, size_t c0, int n, const Cell4<T>* __restrict__ U, const int* __restrict__ perm,
                                 double gma, int prims, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T t[4];
    hcfd::ld_cell(U, ps, (int) (c0 + i), t);
    const size_t j = perm[i];
    const double u0 = t[0], u1 = t[1], u2 = t[2], u3 = t[3];
    if (!prims) {
        out[j] = u0; out[(size_t) n + j] = u1; out[2 * (size_t) n + j] = u2; out[3 * (size_t) n + j] = u3;
        return;
    }
    const double q1 = u1 / u0, q2 = u2 / u0;
    out[j] = u0; out[(size_t) n + j] = q1; out[2 * (size_t) n + j] = q2;
    out[3 * (size_t) n + j] = (gma - 1) * (u3 - 0.5 * u0 * (q1 * q1 + q2 * q2));
}

template <class T>
__global__ void arena_iv_kernel(int n, const double* __restrict__ ivu, const int* __restrict__ perm, T* __restrict__ iv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) iv[i] = T(ivu[perm[i]]);
}

// Instance cells (internal order, from arena cell c0) from 4 x n doubles in input numbering.
template <class T>
__global__ void arena_in_kernel(size_t ps, size_t c0, int n, const double* __restrict__ in, const int* __restrict__ perm,
                                Cell4<T>* U) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t j = perm[i];
    const T u[4] = {T(in[j]), T(in[(size_t) n + j]), T(in[2 * (size_t) n + j]), T(in[3 * (size_t) n + j])};
    hcfd::st_cell(U, ps, (int) (c0 + i), u);
}

// dst[k] = c0 + map[src[k]]: input cell numbers -> arena cell numbers.
__global__ void arena_cellmap_kernel(long long n, int c0, const int* __restrict__ map, const int* __restrict__ src,
                                     int* __restrict__ dst) {
    const long long k = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[k] = c0 + map[src[k]];
}

// dst[k] = c0 + src[k]: tile-local halo cell numbers -> arena cell numbers.
__global__ void arena_offset_kernel(long long n, int c0, const int* __restrict__ src, int* __restrict__ dst) {
    const long long k = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[k] = c0 + src[k];
}

}  // namespace


struct hcfd_arena {
    hcfd_arena_params prm{};
    int device = 0, nsm = 0;
    cudaStream_t stream = nullptr;
    int B = 128, W = 3, Wp = 4, Hcap = 112, Fcap = 288;   // staging capacities (admission limit)
    int Hcur = 0, Fcur = 0;                               // largest halo / entries of the active tiles
    bool dirty = false;                                   // the active list changed since the last rebuild
    // Admissions upload and compute on their own stream, so that they overlap the steps of
    // the instances already active; the step stream waits for them (admit_ev) only when the
    // new instances join the active list.
    cudaStream_t astream = nullptr;
    cudaEvent_t admit_ev = nullptr;
    bool admit_pending = false;
    // host copies of the last active-list upload and the event after which they may change
    std::vector<int> tl_host;
    std::vector<int4> act_host;
    std::vector<int4> chunk_host;
    cudaEvent_t list_ev = nullptr;
    bool list_pending = false;
    size_t Ccap = 0, Ecap = 0, HLcap = 0;
    FreeList fc, fe, fh;
    size_t tsz = 8;
    // device arrays
    void* U[2] = {nullptr, nullptr};
    void* phiG = nullptr;
    void* phiF = nullptr;
    void* iv = nullptr;
    short* cslot = nullptr;
    void* tgeo = nullptr;
    unsigned* tmeta = nullptr;              // pack_meta words
    int* halo = nullptr;
    double* inst_dt = nullptr;
    unsigned long long* inst_dtmin = nullptr;
    hcfd::BCTable* inst_bc = nullptr;
    hcfd::StepStats* stats = nullptr;
    int4* tiles = nullptr;
    int4* act = nullptr;
    int4* chunks = nullptr;                 // residual chunks of the active instances
    double* chunk_r2 = nullptr;
    int* chunk_bad = nullptr;
    size_t chunks_cap = 0;
    int nchunks = 0;
    double* tile_r2 = nullptr;
    int* tile_bad = nullptr;
    unsigned int* err = nullptr;
    int* queue = nullptr;                // pass 1's tile queue (see TileArgs::claim)
    size_t tiles_cap = 0;
    // host
    std::vector<Inst> inst;
    int nact_tiles = 0, nact = 0;
    int cur = 0, par = 0;
    int time_mode = HCFD_GLOBAL_CFL;
    size_t smem1 = 0, smem2 = 0;
    int grid1 = 0, grid2 = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    long long steps_done = 0;
    bool fp32() const { return prm.precision == HCFD_FP32; }
};

// The host half of an admission (hcfd_arena_prepare): everything that does not depend on
// where in the arena the mesh lands.  The mesh arrays are the caller's.
struct hcfd_admission {
    const hcfd_arena* owner = nullptr;
    hcfd_mesh_view mv{};
    int Nc = 0, Nf = 0, F_BC = 0, nreal = 0;
    std::vector<int> cf_off, cf_con, perm, iperm;
    hcfd::TilePlan P;
    hcfd::BCTable bc{};
    double u0[4] = {0, 0, 0, 0};
    double dt = 0;
};

namespace {

void free_graph(hcfd_arena* a) {
    if (a->graph) { cudaGraphExecDestroy(a->graph); a->graph = nullptr; a->graph_steps = 0; }
}

// Orders the step stream after every admission enqueued so far (device-side wait).
int wait_admissions(hcfd_arena* A) {
    if (A->admit_pending) {
        CK(cudaStreamWaitEvent(A->stream, A->admit_ev, 0));
        A->admit_pending = false;
    }
    return HCFD_OK;
}

template <class T>
hcfd::TileArgs<T> arena_args(hcfd_arena* A, int cur, int par) {
    hcfd::TileArgs<T> a{};
    hcfd::StepArgs<T>& s = a.s;
    s.U = (const Cell4<T>*) A->U[cur];
    s.Unew = (Cell4<T>*) A->U[1 - cur];
    s.phiG = (hcfd::Grad8<T>*) A->phiG;
    s.iv = (const T*) A->iv;
    s.Nc = (int) A->Ccap;
    s.limiter = A->prm.limiter;
    s.time_mode = A->time_mode;
    s.gma = T(A->prm.gma);
    s.venkat_K = T(A->prm.venkat_K);
    s.phiF = (Cell4<T>*) A->phiF;
    s.freeze_after = A->prm.freeze_limiter_after;
    a.inst_stats = A->stats;
    a.tgeo = (const T*) A->tgeo;
    a.rec = 8;                             // one plan serves both passes: pass 1 reads If
    a.tmeta = A->tmeta;
    a.halo = A->halo;
    a.cslot = A->cslot;
    a.ntiles = A->nact_tiles;
    a.B = A->B;
    a.Wp = A->Wp;
    a.Hmax = A->Hcur;
    a.Fmax = A->Fcur;
    a.nentries = (long long) A->Ecap;
    a.nhalo = (long long) A->HLcap;
    a.ncap = (long long) A->Ccap;
    a.err = A->err;
    a.polls = 1u << 22;
    a.skip_tile = -1;
    a.ps = (int) A->Ccap;
    a.tiles = A->tiles;
    a.inst_dt = A->inst_dt;
    a.inst_dtmin = A->inst_dtmin;
    a.inst_bc = A->inst_bc;
    a.tile_r2 = A->tile_r2;
    a.tile_bad = A->tile_bad;
    a.par = par;
    return a;
}

template <class T, int W>
int enqueue_step(hcfd_arena* A, int cur, int par) {
    hcfd::TileArgs<T> a = arena_args<T>(A, cur, par);
    constexpr bool COMP = std::is_same<T, float>::value;
    // pass 1 takes its tiles from a queue (per-instance dt minima are order-free), and pass 2,
    // which runs between two pass-1 launches, zeroes it; pass 2 takes every grid-th tile
    // (measured faster for it than a queue)
    a.claim = A->queue;
    a.claim_reset = nullptr;
    hcfd::tile_pass1_kernel<T, W, true><<<A->grid1, A->B + 32, A->smem1, A->stream>>>(a);
    a.claim = nullptr;
    a.claim_reset = A->queue;
    hcfd::tile_pass2_kernel<T, W, COMP, true><<<A->grid2, A->B + 32, A->smem2, A->stream>>>(a);
    arena_chunk_kernel<<<A->nchunks, 256, 0, A->stream>>>(A->chunks, A->tile_r2, A->tile_bad, A->chunk_r2, A->chunk_bad);
    arena_finalize_kernel<<<(A->nact + 127) / 128, 128, 0, A->stream>>>(A->nact, A->nchunks, A->act, A->chunk_r2,
                                                                       A->chunk_bad, A->inst_dt, A->inst_dtmin, A->stats,
                                                                       A->time_mode, par);
    CK(cudaGetLastError());
    return HCFD_OK;
}

template <class T>
int enqueue_step_w(hcfd_arena* A, int cur, int par) {
    return A->W == 3 ? enqueue_step<T, 3>(A, cur, par) : enqueue_step<T, 4>(A, cur, par);
}

template <class T, int W>
int setup_kernels(hcfd_arena* A) {
    constexpr bool COMP = std::is_same<T, float>::value;
    // the attributes allow the largest staging the arena admits; launches size the shared
    // memory to the active instances (configure_kernels)
    const size_t s1 = hcfd::TileSmem<T>(A->B, A->Hcap, A->Fcap, W, A->Wp, false).total;
    const size_t s2 = hcfd::TileSmem<T>(A->B, A->Hcap, A->Fcap, W, A->Wp, true).total;
    int maxsm = 0;
    CK(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, A->device));
    if ((int) s2 > maxsm || (int) s1 > maxsm) return fail(HCFD_EINVAL, "arena: tile does not fit in shared memory");
    CK(cudaFuncSetAttribute(hcfd::tile_pass1_kernel<T, W, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) s1));
    CK(cudaFuncSetAttribute(hcfd::tile_pass2_kernel<T, W, COMP, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) s2));
    return HCFD_OK;
}

// Shared memory and persistent grids for the current staging sizes (Hcur, Fcur): staging
// sized to the active instances rather than to the admission limit lets more CTAs share
// an SM.
template <class T, int W>
int configure_kernels(hcfd_arena* A) {
    constexpr bool COMP = std::is_same<T, float>::value;
    A->smem1 = hcfd::TileSmem<T>(A->B, A->Hcur, A->Fcur, W, A->Wp, false).total;
    A->smem2 = hcfd::TileSmem<T>(A->B, A->Hcur, A->Fcur, W, A->Wp, true).total;
    int b1 = 0, b2 = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, hcfd::tile_pass1_kernel<T, W, true>, A->B + 32, A->smem1));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, hcfd::tile_pass2_kernel<T, W, COMP, true>, A->B + 32, A->smem2));
    if (b1 < 1 || b2 < 1) return fail(HCFD_EINVAL, "arena: kernels cannot be resident");
    A->grid1 = b1 * A->nsm;
    A->grid2 = b2 * A->nsm;
    return HCFD_OK;
}

int configure(hcfd_arena* A) {
    return A->fp32() ? (A->W == 3 ? configure_kernels<float, 3>(A) : configure_kernels<float, 4>(A))
                     : (A->W == 3 ? configure_kernels<double, 3>(A) : configure_kernels<double, 4>(A));
}

// Rebuilds the active tile list and the per-instance tile ranges, in slot order.
int rebuild_active(hcfd_arena* A) {
    int rc = wait_admissions(A);
    if (rc) return rc;
    // the previous upload must have read the host copies before they change
    if (A->list_pending) CK(cudaEventSynchronize(A->list_ev));
    std::vector<int>& tl = A->tl_host;
    std::vector<int4>& act = A->act_host;
    std::vector<int4>& chk = A->chunk_host;
    chk.clear();
    const int nw = A->B / 32;
    tl.clear();
    act.clear();
    int hmax = 0, fmax = 4;
    for (size_t k = 0; k < A->inst.size(); k++) {
        const Inst& I = A->inst[k];
        if (!I.active) continue;
        const int t0 = (int) (tl.size() / 8);
        hmax = std::max(hmax, I.Hmax);
        fmax = std::max(fmax, I.Fmax);
        tl.insert(tl.end(), I.tiles.begin(), I.tiles.end());
        const int t1 = (int) (tl.size() / 8);
        act.push_back(make_int4((int) k, t0, t1, (int) chk.size()));
        for (int p = t0 * nw; p < t1 * nw; p += kChunk)
            chk.push_back(make_int4((int) act.size() - 1, p, std::min(p + kChunk, t1 * nw), 0));
    }
    A->nact_tiles = (int) (tl.size() / 8);
    A->nact = (int) act.size();
    if ((size_t) A->nact_tiles > A->tiles_cap) return fail(HCFD_EINVAL, "arena: tile list capacity exceeded");
    // stream-ordered after the steps already enqueued, before the next ones
    if (!tl.empty()) CK(cudaMemcpyAsync(A->tiles, tl.data(), sizeof(int) * tl.size(), cudaMemcpyHostToDevice, A->stream));
    if (!act.empty()) CK(cudaMemcpyAsync(A->act, act.data(), sizeof(int4) * act.size(), cudaMemcpyHostToDevice, A->stream));
    if (chk.size() > A->chunks_cap) return fail(HCFD_EINVAL, "arena: residual chunk capacity exceeded");
    A->nchunks = (int) chk.size();
    if (!chk.empty()) CK(cudaMemcpyAsync(A->chunks, chk.data(), sizeof(int4) * chk.size(), cudaMemcpyHostToDevice, A->stream));
    CK(cudaEventRecord(A->list_ev, A->stream));
    A->list_pending = true;
    free_graph(A);
    A->Hcur = hmax;
    A->Fcur = fmax;
    A->dirty = false;
    return configure(A);
}

template <class P>
int dalloc(P** p, size_t n) {
    cudaError_t e = cudaMalloc((void**) p, std::max<size_t>(n, 1) * sizeof(P));
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(e == cudaErrorMemoryAllocation ? HCFD_ENOMEM : HCFD_ECUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    return HCFD_OK;
}

void arena_free(hcfd_arena* A) {
    if (!A) return;
    cudaSetDevice(A->device);
    if (A->astream) cudaStreamSynchronize(A->astream);
    if (A->stream) cudaStreamSynchronize(A->stream);
    free_graph(A);
    for (auto& I : A->inst) if (I.d_perm) cudaFree(I.d_perm);
    if (A->admit_ev) cudaEventDestroy(A->admit_ev);
    if (A->list_ev) cudaEventDestroy(A->list_ev);
    if (A->astream) cudaStreamDestroy(A->astream);
    void* p[] = {A->U[0], A->U[1], A->phiG, A->phiF, A->iv, A->cslot, A->tgeo, A->tmeta, A->halo, A->inst_dt, A->inst_dtmin,
                 A->inst_bc, A->stats, A->tiles, A->act, A->tile_r2, A->tile_bad, A->err, A->queue, A->chunks,
                 A->chunk_r2, A->chunk_bad};
    for (void* q : p) if (q) cudaFree(q);
    if (A->stream) cudaStreamDestroy(A->stream);
}

void prim_to_cons(const double* q, double gma, double* u) {
    u[0] = q[0];
    for (int v = 1; v < 4; v++) u[v] = q[0] * q[v];
    u[3] = q[3] / (gma - 1) + 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2]);
}

}  // namespace

extern "C" {

int hcfd_arena_create(const hcfd_arena_params* prm, hcfd_arena** out) {
    hcfd::clear_error();
    if (!prm || !out) return fail(HCFD_EINVAL, "arena_create: null argument");
    *out = nullptr;
    const hcfd_arena_params& p = *prm;
    if (p.hbm_budget < ((size_t) 16 << 20) || !(p.gma > 1.0) || (p.precision != HCFD_FP64 && p.precision != HCFD_FP32) ||
        (p.limiter != HCFD_LIMITER_BJ && p.limiter != HCFD_LIMITER_VENKAT) || p.max_instances < 1 ||
        p.max_instances > 65536 || p.tile < 0 || p.tile > 256 || (p.tile % 32) || (p.slots != 0 && p.slots != 3 && p.slots != 4) ||
        (p.time_mode != HCFD_FIXED_DT && p.time_mode != HCFD_GLOBAL_CFL && p.time_mode != HCFD_LOCAL_CFL) ||
        p.freeze_limiter_after < 0)
        return fail(HCFD_EINVAL, "arena_create: bad parameters");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(HCFD_ECUDA, "arena_create: no CUDA device");
    auto A = std::make_unique<hcfd_arena>();
    A->prm = p;
    CK(cudaGetDevice(&A->device));
    CK(cudaDeviceGetAttribute(&A->nsm, cudaDevAttrMultiProcessorCount, A->device));
    A->B = p.tile ? p.tile : 128;
    A->W = p.slots == 4 ? 4 : 3;
    A->Wp = A->W;
    A->time_mode = p.time_mode;
    // per-tile staging capacities (generous for triangle and quad meshes at this tile size)
    A->Hcap = A->B * 7 / 8 + 16;
    A->Fcap = A->B * 9 / 4 + 16;
    A->tsz = A->fp32() ? 4 : 8;
    const size_t ts = A->tsz;
    // Budget split, bytes per cell: state x2, gradients, iv, slots; ~1.75 face entries per
    // cell (records + metadata) and ~0.6 halo ids per cell, as the wedge meshes need.
    const double per_cell = 2 * 4 * ts + 8 * ts + ts + A->Wp * 2 + 1.75 * (8 * ts + 8) + 0.6 * 4 +
                            (p.freeze_limiter_after > 0 ? 4 * ts : 0);
    size_t budget = p.hbm_budget;
    size_t C = (size_t) (budget / per_cell);
    C = std::min<size_t>(C, (size_t) 1 << 30);   // cell indices stay within int
    C = (C / A->B) * A->B;
    if (C < (size_t) A->B) return fail(HCFD_EINVAL, "arena_create: budget below one tile");
    A->Ccap = C;
    A->Ecap = (size_t) (1.75 * C) / 4 * 4;
    A->HLcap = (size_t) (0.6 * C);
    A->tiles_cap = C / A->B;
    A->chunks_cap = A->tiles_cap * (A->B / 32) / kChunk + p.max_instances + 1;
    A->fc.init(C / A->B);
    A->fe.init(A->Ecap / 4);
    A->fh.init(A->HLcap);
    A->inst.resize(p.max_instances);
    CK(cudaStreamCreateWithFlags(&A->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&A->astream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&A->admit_ev, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&A->list_ev, cudaEventDisableTiming));
    hcfd_arena* h = A.get();
    auto bail = [&](int code) { arena_free(h); A.release(); delete h; return code; };
    int rc;
    if ((rc = dalloc((char**) &h->U[0], 4 * ts * C)) || (rc = dalloc((char**) &h->U[1], 4 * ts * C)) ||
        (rc = dalloc((char**) &h->phiG, 8 * ts * C)) || (rc = dalloc((char**) &h->iv, ts * C)) ||
        (p.freeze_limiter_after > 0 && (rc = dalloc((char**) &h->phiF, 4 * ts * C))) ||
        (rc = dalloc(&h->cslot, h->Wp * C)) || (rc = dalloc((char**) &h->tgeo, 8 * ts * h->Ecap)) ||
        (rc = dalloc(&h->tmeta, h->Ecap)) || (rc = dalloc(&h->halo, h->HLcap)) ||
        (rc = dalloc(&h->inst_dt, p.max_instances)) || (rc = dalloc(&h->inst_dtmin, 2 * (size_t) p.max_instances)) ||
        (rc = dalloc(&h->inst_bc, p.max_instances)) || (rc = dalloc(&h->stats, p.max_instances)) ||
        (rc = dalloc(&h->tiles, 2 * h->tiles_cap)) || (rc = dalloc(&h->act, p.max_instances)) ||
        (rc = dalloc(&h->tile_r2, h->tiles_cap * (h->B / 32))) || (rc = dalloc(&h->tile_bad, h->tiles_cap * (h->B / 32))) ||
        (rc = dalloc(&h->err, 1)) || (rc = dalloc(&h->queue, 1)) || (rc = dalloc(&h->chunks, h->chunks_cap)) ||
        (rc = dalloc(&h->chunk_r2, h->chunks_cap)) || (rc = dalloc(&h->chunk_bad, h->chunks_cap)))
        return bail(rc);
    cudaError_t ce = cudaMemsetAsync(h->err, 0, sizeof(unsigned int), h->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->queue, 0, sizeof(int), h->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->U[0], 0, 4 * ts * C, h->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->U[1], 0, 4 * ts * C, h->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->phiG, 0, 8 * ts * C, h->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->iv, 0, ts * C, h->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->stream);
    if (ce != cudaSuccess) return bail(fail(HCFD_ECUDA, std::string("arena_create: ") + cudaGetErrorString(ce)));
    rc = h->fp32() ? (h->W == 3 ? setup_kernels<float, 3>(h) : setup_kernels<float, 4>(h))
                   : (h->W == 3 ? setup_kernels<double, 3>(h) : setup_kernels<double, 4>(h));
    if (rc) return bail(rc);
    *out = A.release();
    return HCFD_OK;
}

int hcfd_arena_prepare(const hcfd_arena* A, const hcfd_mesh_view* mv, const int* bcmap, int nbcmap, const double* qbc,
                       const double* qic, double dt_or_cfl, hcfd_admission** out) {
    hcfd::clear_error();
    if (!A || !mv || !bcmap || !qbc || !qic || !out || !(dt_or_cfl > 0)) return fail(HCFD_EINVAL, "arena_prepare: bad argument");
    *out = nullptr;
    int rc = hcfd::validate_view(*mv);
    if (rc) return rc;
    auto D = std::make_unique<hcfd_admission>();
    D->owner = A;
    D->mv = *mv;
    const int Nc = mv->Nc, Nf = mv->Nf, Ncol = mv->Ncol, NBC = mv->NBCcol;
    if (NBC > hcfd::MAXBC) return fail(HCFD_EINVAL, "arena_prepare: more than 16 boundary colours");
    const int F_BC = mv->coloff[Ncol - NBC];
    hcfd::build_cf(Nc, Nf, mv->fc_con, D->cf_off, D->cf_con);
    std::vector<char> ghost(Nc, 0);
    for (int f = F_BC; f < Nf; f++) ghost[mv->fc_con[2 * f + 1]] = 1;
    int nreal = 0, maxdeg = 0;
    for (int c = 0; c < Nc; c++) if (!ghost[c]) { nreal++; maxdeg = std::max(maxdeg, D->cf_off[c + 1] - D->cf_off[c]); }
    if (maxdeg > A->W) return fail(HCFD_EINVAL, "arena_prepare: cells with more faces than the arena's slots");
    D->perm = hcfd::morton_order(*mv);
    D->iperm.resize(Nc);
    for (int i = 0; i < Nc; i++) D->iperm[D->perm[i]] = i;
    std::vector<int> bc_first;
    for (int col = Ncol - NBC; col < Ncol; col++) bc_first.push_back(mv->coloff[col]);
    rc = hcfd::build_tile_plan(*mv, D->cf_off, D->cf_con, ghost, D->perm, F_BC, bc_first, A->B, A->W, D->P);
    if (rc) return rc;
    if (D->P.Hmax > A->Hcap || D->P.Fmax > A->Fcap)
        return fail(HCFD_EINVAL, "arena_prepare: a tile's halo or faces exceed the arena's staging capacity");
    // BC table (Euler::gather_BCs, src/Base/Euler.cpp:42-60)
    hcfd::BCTable& bc = D->bc;
    bc = hcfd::BCTable{};
    bc.nbc = NBC;
    for (int col = Ncol - NBC; col < Ncol; col++) {
        const int b = col - (Ncol - NBC), tag = mv->coltag[col];
        if (tag < 0 || tag >= nbcmap || bcmap[tag] < HCFD_SYMMETRY || bcmap[tag] > HCFD_SUBOUTLET)
            return fail(HCFD_EINVAL, "arena_prepare: bad BC map");
        bc.type[b] = bcmap[tag];
        bc.F1[b] = mv->coloff[col];
        for (int v = 0; v < 4; v++) bc.QBC[b][v] = qbc[4 * b + v];
        prim_to_cons(bc.QBC[b], A->prm.gma, bc.UBC[b]);
    }
    bc.F1[NBC] = Nf;
    // initial state (Euler::initialise, src/Base/Euler.cpp:62-77)
    prim_to_cons(qic, A->prm.gma, D->u0);
    D->Nc = Nc; D->Nf = Nf; D->F_BC = F_BC; D->nreal = nreal;
    D->dt = dt_or_cfl;
    *out = D.release();
    return HCFD_OK;
}

size_t hcfd_admission_cells(const hcfd_admission* D) {
    return D && D->owner ? (size_t) D->P.ntiles * D->owner->B : 0;
}

void hcfd_admission_free(hcfd_admission* D) { delete D; }

int hcfd_arena_admit_prepared(hcfd_arena* A, const hcfd_admission* D, int* slot_out) {
    hcfd::clear_error();
    if (!A || !D || !slot_out) return fail(HCFD_EINVAL, "arena_admit: bad argument");
    if (D->owner != A) return fail(HCFD_EINVAL, "arena_admit: the admission was prepared for another arena");
    CK(cudaSetDevice(A->device));
    int slot = -1;
    for (size_t k = 0; k < A->inst.size(); k++) if (!A->inst[k].active) { slot = (int) k; break; }
    if (slot < 0) return fail(HCFD_EAGAIN, "arena_admit: all instance slots in use");
    const hcfd_mesh_view* mv = &D->mv;
    const hcfd::TilePlan& P = D->P;
    const int Nc = D->Nc, Nf = D->Nf, F_BC = D->F_BC;
    // ranges in the arena (budget admission)
    Inst I;
    I.Nc = Nc; I.Nf = Nf; I.Nreal = D->nreal; I.ntiles = P.ntiles; I.Hmax = P.Hmax; I.Fmax = P.Fmax;
    I.ncell = (size_t) P.ntiles * A->B;
    I.ne = P.efid.size();
    I.nh = P.halo.size();
    size_t ct = 0, eo = 0, ho = 0;
    if (!A->fc.alloc(P.ntiles, ct)) return fail(HCFD_EAGAIN, "arena_admit: cell capacity exhausted");
    if (!A->fe.alloc(I.ne / 4, eo)) { A->fc.release(ct, P.ntiles); return fail(HCFD_EAGAIN, "arena_admit: face capacity exhausted"); }
    if (!A->fh.alloc(I.nh, ho)) {
        A->fc.release(ct, P.ntiles); A->fe.release(eo, I.ne / 4);
        return fail(HCFD_EAGAIN, "arena_admit: halo capacity exhausted");
    }
    I.c0 = ct * A->B; I.e0 = eo * 4; I.h0 = ho;
    auto undo = [&]() { A->fc.release(ct, P.ntiles); A->fe.release(eo, I.ne / 4); A->fh.release(ho, I.nh); };
    // tile descriptors with arena offsets
    I.tiles.resize(8 * (size_t) P.ntiles);
    for (int t = 0; t < P.ntiles; t++) {
        int* d = &I.tiles[8 * (size_t) t];
        d[0] = (int) (I.c0 + (size_t) t * A->B);
        d[1] = (int) (I.e0 + P.foff[t]);
        d[2] = P.foff[t + 1] - P.foff[t];
        d[3] = slot;
        d[4] = (int) (I.h0 + P.hoff[t]);
        d[5] = P.hoff[t + 1] - P.hoff[t];
        d[6] = d[7] = 0;
    }
    // device work: geometry of this mesh (stream-ordered temporaries), then the arena ranges
    cudaStream_t st = A->astream;
    int *d_fn = nullptr, *d_fcu = nullptr, *d_fcg = nullptr, *d_cnoff = nullptr, *d_cncon = nullptr, *d_cfoff = nullptr,
        *d_cfcon = nullptr, *d_efid = nullptr, *d_foff = nullptr, *d_iperm = nullptr, *d_halo = nullptr;
    double *d_nodes = nullptr, *d_xc = nullptr, *d_ivu = nullptr;
    hcfd::FaceGeo<double>* d_geo = nullptr;
    const int ncn = mv->cn_off[Nc];
    cudaError_t ce = cudaSuccess;
    auto tmp = [&](auto** p, size_t n) {
        if (ce == cudaSuccess) ce = cudaMallocAsync((void**) p, std::max<size_t>(n, 1) * sizeof(**p), st);
    };
    tmp(&d_fn, 2 * (size_t) Nf); tmp(&d_fcu, 2 * (size_t) Nf); tmp(&d_fcg, 2 * (size_t) Nf);
    tmp(&d_cnoff, Nc + 1); tmp(&d_cncon, ncn); tmp(&d_cfoff, Nc + 1); tmp(&d_cfcon, D->cf_con.size());
    tmp(&d_efid, I.ne); tmp(&d_foff, P.foff.size()); tmp(&d_iperm, Nc); tmp(&d_halo, I.nh);
    tmp(&d_nodes, 2 * (size_t) mv->Nn); tmp(&d_xc, 2 * (size_t) Nc); tmp(&d_ivu, Nc); tmp(&d_geo, Nf);
    auto tmp_free = [&]() {
        void* t[] = {d_fn, d_fcu, d_fcg, d_cnoff, d_cncon, d_cfoff, d_cfcon, d_efid, d_foff, d_iperm, d_halo,
                     d_nodes, d_xc, d_ivu, d_geo};
        for (void* q : t) if (q) cudaFreeAsync(q, st);
    };
    if (ce == cudaSuccess) ce = cudaMallocAsync((void**) &I.d_perm, sizeof(int) * (size_t) Nc, st);
    if (ce != cudaSuccess) {
        tmp_free();
        if (I.d_perm) cudaFreeAsync(I.d_perm, st);
        cudaStreamSynchronize(st);
        undo();
        return fail(ce == cudaErrorMemoryAllocation ? HCFD_ENOMEM : HCFD_ECUDA,
                    std::string("arena_admit: ") + cudaGetErrorString(ce));
    }
    auto up = [&](void* dst, const void* src, size_t bytes) {
        if (ce == cudaSuccess && bytes) ce = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
    };
    up(d_fn, mv->fn_con, 8 * (size_t) Nf);
    up(d_fcu, mv->fc_con, 8 * (size_t) Nf);
    up(d_cnoff, mv->cn_off, 4 * (size_t) (Nc + 1));
    up(d_cncon, mv->cn_con, 4 * (size_t) ncn);
    up(d_cfoff, D->cf_off.data(), 4 * D->cf_off.size());
    up(d_cfcon, D->cf_con.data(), 4 * D->cf_con.size());
    up(d_efid, P.efid.data(), 4 * I.ne);
    up(d_foff, P.foff.data(), 4 * P.foff.size());
    up(d_iperm, D->iperm.data(), 4 * (size_t) Nc);
    up(d_halo, P.halo.data(), 4 * I.nh);
    up(d_nodes, mv->nodes, 16 * (size_t) mv->Nn);
    up(I.d_perm, D->perm.data(), 4 * (size_t) Nc);
    const std::vector<unsigned> mw = hcfd::packed_meta(P);
    up(A->tmeta + I.e0, mw.data(), 4 * mw.size());
    up(A->cslot + A->Wp * I.c0, P.cslot.data(), 2 * P.cslot.size());
    if (ce == cudaSuccess) {
        arena_cellmap_kernel<<<nblk(2 * (long long) Nf, 256), 256, 0, st>>>(2 * (long long) Nf, (int) I.c0, d_iperm, d_fcu, d_fcg);
        if (I.nh) arena_offset_kernel<<<nblk((long long) I.nh, 256), 256, 0, st>>>((long long) I.nh, (int) I.c0, d_halo, A->halo + I.h0);
        hcfd::geom_xc_kernel<<<nblk(Nc, 256), 256, 0, st>>>(Nc, d_cnoff, d_cncon, d_nodes, d_xc);
        hcfd::geom_face_kernel<<<nblk(Nf, 256), 256, 0, st>>>(Nf, F_BC, d_fn, d_fcu, d_nodes, d_xc, d_geo);
        hcfd::geom_iv_kernel<<<nblk(Nc, 256), 256, 0, st>>>(Nc, F_BC, d_cfoff, d_cfcon, d_fcu, d_geo, d_ivu);
        ce = cudaMemsetAsync((char*) A->iv + A->tsz * I.c0, 0, A->tsz * I.ncell, st);
        if (A->fp32()) {
            arena_iv_kernel<float><<<nblk(Nc, 256), 256, 0, st>>>(Nc, d_ivu, I.d_perm, (float*) A->iv + I.c0);
            hcfd::gather_geo_kernel<float><<<P.ntiles, 128, 0, st>>>(P.ntiles, d_foff, d_efid, d_geo, (float*) A->tgeo + 8 * I.e0, 8);
        } else {
            arena_iv_kernel<double><<<nblk(Nc, 256), 256, 0, st>>>(Nc, d_ivu, I.d_perm, (double*) A->iv + I.c0);
            hcfd::gather_geo_kernel<double><<<P.ntiles, 128, 0, st>>>(P.ntiles, d_foff, d_efid, d_geo, (double*) A->tgeo + 8 * I.e0, 8);
        }
        // initial state into the current buffer, then the ghost cells from the BCs
        const double* u = D->u0;
        const int nfill = (int) I.ncell;
        if (A->fp32()) {
            arena_fill_kernel<float><<<nblk(nfill, 256), 256, 0, st>>>(A->Ccap, I.c0, nfill, (Cell4<float>*) A->U[A->cur], u[0], u[1], u[2], u[3]);
            if (Nf > F_BC)
                hcfd::bc_cells_kernel<float><<<nblk(Nf - F_BC, 256), 256, 0, st>>>((int) A->Ccap, Nf, F_BC, d_fcg, d_geo,
                                                                                   (Cell4<float>*) A->U[A->cur], float(A->prm.gma), D->bc);
        } else {
            arena_fill_kernel<double><<<nblk(nfill, 256), 256, 0, st>>>(A->Ccap, I.c0, nfill, (Cell4<double>*) A->U[A->cur], u[0], u[1], u[2], u[3]);
            if (Nf > F_BC)
                hcfd::bc_cells_kernel<double><<<nblk(Nf - F_BC, 256), 256, 0, st>>>((int) A->Ccap, Nf, F_BC, d_fcg, d_geo,
                                                                                    (Cell4<double>*) A->U[A->cur], A->prm.gma, D->bc);
        }
        if (ce == cudaSuccess) ce = cudaGetLastError();
    }
    const unsigned long long infb[2] = {0x7FF0000000000000ULL, 0x7FF0000000000000ULL};
    up(A->inst_dtmin + 2 * slot, infb, sizeof(infb));
    up(A->inst_dt + slot, &D->dt, sizeof(double));
    up(A->inst_bc + slot, &D->bc, sizeof(hcfd::BCTable));
    if (ce == cudaSuccess) ce = cudaMemsetAsync(A->stats + slot, 0, sizeof(hcfd::StepStats), st);
    tmp_free();
    // Host sources are pageable (the stack included): each upload has copied its source by the
    // time it returns.  The device work goes on behind the steps already enqueued; the step
    // stream waits for it when the active list next changes.
    if (ce == cudaSuccess) ce = cudaEventRecord(A->admit_ev, st);
    if (ce != cudaSuccess) {
        cudaStreamSynchronize(st);
        cudaFree(I.d_perm);
        undo();
        return fail(HCFD_ECUDA, std::string("arena_admit: ") + cudaGetErrorString(ce));
    }
    A->admit_pending = true;
    I.dt = D->dt;
    I.active = true;
    I.admitted_step = A->steps_done;
    A->inst[slot] = std::move(I);
    A->dirty = true;     // the active list is rebuilt once before the next step, however many are admitted
    *slot_out = slot;
    return HCFD_OK;
}

int hcfd_arena_admit(hcfd_arena* A, const hcfd_mesh_view* mv, const int* bcmap, int nbcmap, const double* qbc,
                     const double* qic, double dt_or_cfl, int* slot_out) {
    hcfd_admission* D = nullptr;
    int rc = hcfd_arena_prepare(A, mv, bcmap, nbcmap, qbc, qic, dt_or_cfl, &D);
    if (rc) return rc;
    rc = hcfd_arena_admit_prepared(A, D, slot_out);
    hcfd_admission_free(D);
    return rc;
}

int hcfd_arena_step(hcfd_arena* A, int nsteps) {
    hcfd::clear_error();
    if (!A || nsteps < 0) return fail(HCFD_EINVAL, "arena_step: bad argument");
    CK(cudaSetDevice(A->device));
    if (A->dirty) {
        const int rc = rebuild_active(A);
        if (rc) return rc;
    }
    if (A->nact == 0 || nsteps == 0) return HCFD_OK;
    // one graph holds two steps (the ping-pong buffers and dt slots return to their start)
    if (!A->graph) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(A->stream, cudaStreamCaptureModeThreadLocal));
        int rc = HCFD_OK;
        for (int k = 0; k < 2 && rc == HCFD_OK; k++)
            rc = A->fp32() ? enqueue_step_w<float>(A, A->cur ^ k, A->par ^ k) : enqueue_step_w<double>(A, A->cur ^ k, A->par ^ k);
        cudaError_t e = cudaStreamEndCapture(A->stream, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return fail(HCFD_ECUDA, std::string("arena_step: capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&A->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(HCFD_ECUDA, std::string("arena_step: instantiate: ") + cudaGetErrorString(e));
        A->graph_steps = 2;
    }
    int n = nsteps;
    while (n >= 2) {
        CK(cudaGraphLaunch(A->graph, A->stream));
        n -= 2;
    }
    if (n == 1) {
        int rc = A->fp32() ? enqueue_step_w<float>(A, A->cur, A->par) : enqueue_step_w<double>(A, A->cur, A->par);
        if (rc) return rc;
        A->cur ^= 1;
        A->par ^= 1;
        free_graph(A);   // the graph was captured for the other parity
    }
    A->steps_done += nsteps;
    return HCFD_OK;
}

int hcfd_arena_poll(hcfd_arena* A, int max, int* slots, hcfd_step_stats* stats, int* n) {
    hcfd::clear_error();
    if (!A || !n || max < 0 || (max > 0 && (!slots || !stats))) return fail(HCFD_EINVAL, "arena_poll: bad argument");
    CK(cudaSetDevice(A->device));
    {
        const int rc_ = wait_admissions(A);
        if (rc_) return rc_;
    }
    std::vector<hcfd::StepStats> st(A->inst.size());
    unsigned int err = 0;
    CK(cudaMemcpyAsync(st.data(), A->stats, sizeof(hcfd::StepStats) * st.size(), cudaMemcpyDeviceToHost, A->stream));
    CK(cudaMemcpyAsync(&err, A->err, sizeof(err), cudaMemcpyDeviceToHost, A->stream));
    CK(cudaStreamSynchronize(A->stream));
    int k = 0;
    for (size_t i = 0; i < A->inst.size() && k < max; i++) {
        const Inst& I = A->inst[i];
        if (!I.active) continue;
        slots[k] = (int) i;
        stats[k].dt = st[i].dt_last;
        stats[k].res_l2 = I.Nreal ? std::sqrt(st[i].res2_last / I.Nreal) : 0.0;
        stats[k].res_first = I.Nreal ? std::sqrt(st[i].res2_first / I.Nreal) : 0.0;
        stats[k].steps = st[i].steps;
        stats[k].nonfinite = st[i].nonfinite;
        k++;
    }
    *n = k;
    if (err & 4u) return fail(HCFD_EINVAL, "arena, checked build: a tile index was out of range (corrupt tile plan)");
    if (err) return fail(HCFD_ETIMEOUT, "arena: a bounded device wait gave up");
    return HCFD_OK;
}

int hcfd_arena_fetch(hcfd_arena* A, int slot, int prims, double* const* out) {
    hcfd::clear_error();
    if (!A || slot < 0 || slot >= (int) A->inst.size() || !A->inst[slot].active || !out)
        return fail(HCFD_EINVAL, "arena_fetch: bad argument");
    CK(cudaSetDevice(A->device));
    {
        const int rc_ = wait_admissions(A);
        if (rc_) return rc_;
    }
    const Inst& I = A->inst[slot];
    double* d_out = nullptr;
    CK(cudaMallocAsync((void**) &d_out, sizeof(double) * 4 * (size_t) I.Nc, A->stream));
    if (A->fp32())
        arena_out_kernel<float><<<nblk(I.Nc, 256), 256, 0, A->stream>>>(A->Ccap, I.c0, I.Nc, (const Cell4<float>*) A->U[A->cur], I.d_perm, A->prm.gma, prims, d_out);
    else
        arena_out_kernel<double><<<nblk(I.Nc, 256), 256, 0, A->stream>>>(A->Ccap, I.c0, I.Nc, (const Cell4<double>*) A->U[A->cur], I.d_perm, A->prm.gma, prims, d_out);
    cudaError_t e = cudaGetLastError();
    for (int v = 0; v < 4 && e == cudaSuccess; v++)
        e = cudaMemcpyAsync(out[v], d_out + (size_t) v * I.Nc, sizeof(double) * I.Nc, cudaMemcpyDeviceToHost, A->stream);
    cudaFreeAsync(d_out, A->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(A->stream);
    if (e != cudaSuccess) return fail(HCFD_ECUDA, std::string("arena_fetch: ") + cudaGetErrorString(e));
    return HCFD_OK;
}

// One instance's exact snapshot, in the file format of hcfd_gpu_checkpoint.
int hcfd_arena_checkpoint(hcfd_arena* A, int slot, const char* path) {
    hcfd::clear_error();
    if (!A || slot < 0 || slot >= (int) A->inst.size() || !A->inst[slot].active || !path)
        return fail(HCFD_EINVAL, "arena_checkpoint: bad argument");
    CK(cudaSetDevice(A->device));
    {
        const int rc_ = wait_admissions(A);
        if (rc_) return rc_;
    }
    const Inst& I = A->inst[slot];
    const size_t n = 4 * (size_t) I.Nc;
    const bool frz = A->phiF != nullptr;
    std::vector<double> U(n), phi(frz ? n : 0);
    hcfd::StepStats st{};
    double* d_out = nullptr;
    CK(cudaMallocAsync((void**) &d_out, sizeof(double) * n, A->stream));
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < (frz ? 2 : 1) && e == cudaSuccess; k++) {
        const void* src = k == 0 ? A->U[A->cur] : A->phiF;
        if (A->fp32())
            arena_out_kernel<float><<<nblk(I.Nc, 256), 256, 0, A->stream>>>(A->Ccap, I.c0, I.Nc, (const Cell4<float>*) src, I.d_perm, A->prm.gma, 0, d_out);
        else
            arena_out_kernel<double><<<nblk(I.Nc, 256), 256, 0, A->stream>>>(A->Ccap, I.c0, I.Nc, (const Cell4<double>*) src, I.d_perm, A->prm.gma, 0, d_out);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(k == 0 ? U.data() : phi.data(), d_out, sizeof(double) * n, cudaMemcpyDeviceToHost, A->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(A->stream);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&st, A->stats + slot, sizeof(st), cudaMemcpyDeviceToHost, A->stream);
    cudaFreeAsync(d_out, A->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(A->stream);
    if (e != cudaSuccess) return fail(HCFD_ECUDA, std::string("arena_checkpoint: ") + cudaGetErrorString(e));
    hcfd::CkptHeader h{};
    std::memcpy(h.magic, "HCFDCKP1", 8);
    h.version = 1;
    h.precision = A->prm.precision;
    h.Nc = I.Nc;
    h.has_phiF = frz ? 1 : 0;
    h.steps = st.steps;
    h.res2_first = st.res2_first;
    h.res2_last = st.res2_last;
    h.dt_last = st.dt_last;
    h.nonfinite = st.nonfinite;
    return hcfd::ckpt_write(path, h, U, frz ? &phi : nullptr);
}

// Restores a checkpoint into an admitted instance of the same mesh (its state, statistics
// and recorded limiter values): its next steps continue the original solve bit for bit.
int hcfd_arena_restore(hcfd_arena* A, int slot, const char* path) {
    hcfd::clear_error();
    if (!A || slot < 0 || slot >= (int) A->inst.size() || !A->inst[slot].active || !path)
        return fail(HCFD_EINVAL, "arena_restore: bad argument");
    CK(cudaSetDevice(A->device));
    {
        const int rc_ = wait_admissions(A);
        if (rc_) return rc_;
    }
    const Inst& I = A->inst[slot];
    hcfd::CkptHeader h;
    std::vector<double> U, phi;
    int rc = hcfd::ckpt_read(path, h, &U, &phi);
    if (rc) return rc;
    const bool frz = A->phiF != nullptr;
    if (h.Nc != I.Nc) return fail(HCFD_EINVAL, "arena_restore: the checkpoint is of a mesh with another cell count");
    if (h.precision != A->prm.precision) return fail(HCFD_EINVAL, "arena_restore: the checkpoint is of another precision");
    if ((h.has_phiF != 0) != frz) return fail(HCFD_EINVAL, "arena_restore: limiter freezing differs");
    const size_t n = 4 * (size_t) I.Nc;
    double* d_in = nullptr;
    CK(cudaMallocAsync((void**) &d_in, sizeof(double) * n, A->stream));
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < (frz ? 2 : 1) && e == cudaSuccess; k++) {
        void* dst = k == 0 ? A->U[A->cur] : A->phiF;
        e = cudaMemcpyAsync(d_in, k == 0 ? U.data() : phi.data(), sizeof(double) * n, cudaMemcpyHostToDevice, A->stream);
        if (e != cudaSuccess) break;
        if (A->fp32()) arena_in_kernel<float><<<nblk(I.Nc, 256), 256, 0, A->stream>>>(A->Ccap, I.c0, I.Nc, d_in, I.d_perm, (Cell4<float>*) dst);
        else arena_in_kernel<double><<<nblk(I.Nc, 256), 256, 0, A->stream>>>(A->Ccap, I.c0, I.Nc, d_in, I.d_perm, (Cell4<double>*) dst);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(A->stream);
    }
    hcfd::StepStats st{};
    st.res2_first = h.res2_first;
    st.res2_last = h.res2_last;
    st.dt_last = h.dt_last;
    st.steps = h.steps;
    st.nonfinite = h.nonfinite;
    if (e == cudaSuccess) e = cudaMemcpyAsync(A->stats + slot, &st, sizeof(st), cudaMemcpyHostToDevice, A->stream);
    cudaFreeAsync(d_in, A->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(A->stream);
    if (e != cudaSuccess) return fail(HCFD_ECUDA, std::string("arena_restore: ") + cudaGetErrorString(e));
    return HCFD_OK;
}

int hcfd_arena_release(hcfd_arena* A, int slot) {
    hcfd::clear_error();
    if (!A || slot < 0 || slot >= (int) A->inst.size() || !A->inst[slot].active) return fail(HCFD_EINVAL, "arena_release: bad slot");
    CK(cudaSetDevice(A->device));
    {
        const int rc_ = wait_admissions(A);
        if (rc_) return rc_;
    }
    CK(cudaStreamSynchronize(A->stream));
    Inst& I = A->inst[slot];
    A->fc.release(I.c0 / A->B, I.ntiles);
    A->fe.release(I.e0 / 4, I.ne / 4);
    A->fh.release(I.h0, I.nh);
    if (I.d_perm) cudaFree(I.d_perm);
    I = Inst();
    A->dirty = true;
    return HCFD_OK;
}

int hcfd_arena_info(hcfd_arena* A, hcfd_arena_info_t* info) {
    if (!A || !info) return fail(HCFD_EINVAL, "arena_info: bad argument");
    if (A->dirty) {
        CK(cudaSetDevice(A->device));
        const int rc = rebuild_active(A);
        if (rc) return rc;
    }
    info->cell_capacity = A->Ccap;
    info->cells_used = A->fc.used * A->B;
    info->face_capacity = A->Ecap;
    info->faces_used = A->fe.used * 4;
    info->active = A->nact;
    info->active_tiles = A->nact_tiles;
    info->steps = A->steps_done;
    info->tile = A->B;
    return HCFD_OK;
}

void hcfd_arena_destroy(hcfd_arena* A) {
    if (!A) return;
    arena_free(A);
    delete A;
}

}  // extern "C"
