// Tiled step kernels: persistent CTAs walk the tiles of the execution plan (hcfd_plan.cpp).
// Per tile, the contiguous blocks (the tile's own cells, its face records and face
// metadata) are staged into shared memory with TMA bulk copies (cp.async.bulk, completion
// on an mbarrier) and the halo cells with 16-byte cp.async gathers; all arithmetic then
// reads shared memory.
//
// pass 1 (thread per tile cell): Green-Gauss gradient, limiter, CFL dt -> phiG (global).
// pass 2: face phase (thread per face entry) computes each face flux once per tile and
//         writes F over the staged face record's two r pairs (the cell phase does not read
//         them); cell phase (thread per tile cell) sums A_f F of its faces in increasing face
//         order, updates the cell and refreshes its ghost cells.
// The arithmetic is that of the thread-per-cell kernels in hcfd_kernels.cuh, operation for
// operation; only where the operands come from differs.
#pragma once
#include "hcfd_internal.hpp"
#include "hcfd_kernels.cuh"

#include <vector>

namespace hcfd {

template <class T>
struct TileArgs {
    StepArgs<T> s;                         // state, stats, BC table, modes
    const T* __restrict__ tgeo;            // face records, per tile pair-major (see ldp), rec values each
    int rec;                               // values per face record: 8, or 7 in a pass-2 plan of its own
    const unsigned* __restrict__ tmeta;    // one word per entry (pack_meta): la, lb, bc
    const int* __restrict__ foff;          // [ntiles + 1], multiples of 4
    const int* __restrict__ hoff;          // [ntiles + 1]
    const int* __restrict__ halo;          // internal cell ids
    const short* __restrict__ cslot;       // [ntiles * B * Wp]: (entry << 1) | cell-is-right, or -1; Wp = W
    int ntiles, B, Wp, Hmax, Fmax;
    unsigned int* err;                     // bit 0: a bounded wait gave up; bit 1: copies did not drain;
                                           // bit 2: an index out of range (checked build)
    unsigned polls;                        // poll limit of every bounded wait (2^22 by default)
    int skip_tile;                         // failure injection for tests: the producer arms nothing
                                           // for this tile (-1: none)
    int ps;                                // plane stride of the cell planes (Nc, or the arena's capacity)
    // Arena mode (many meshes in one flat arena; see hcfd_arena.cu).  Tile i of the active
    // list is described by tiles[2i] = {first cell, first entry, entries, instance} and
    // tiles[2i+1] = {first halo id, halo count, -, -}; every arena tile holds B cells.
    const int4* __restrict__ tiles;
    const double* __restrict__ inst_dt;    // per instance: dt (fixed mode) or CFL number
    unsigned long long* inst_dtmin;        // per instance, two parity slots (double bits)
    const BCTable* __restrict__ inst_bc;   // per instance
    const StepStats* inst_stats;           // per instance (step counts for limiter freezing)
    double* tile_r2;                       // per active tile and compute warp (t * B/32 + warp): sum of R_rho^2
    int* tile_bad;                         // same layout: a NaN/Inf appeared
    int par;                               // which dtmin slot this step uses
    // Tile queue: each CTA takes tile blockIdx.x first, then, with `claim` set, the tile
    // gridDim.x + atomicAdd(claim, 1) (CTAs that finish early take more tiles), else every
    // gridDim.x-th tile.  `claim_reset` (the other pass's queue) is zeroed by this kernel:
    // the other pass runs before and after it in stream order, never during it.
    int* claim;
    int* claim_reset;
    long long nentries, nhalo, ncap;       // lengths of tgeo/tmeta (entries), halo, and of the
                                           // per-cell arrays iv/cslot (cells): checked build
};

// Metadata of a face entry in one 32-bit word: the local index (tile cell 0..B-1, halo cell
// B..) of its left cell in bits 0-12, of its right cell in bits 13-25, and its boundary
// condition's index + 1 in bits 26-30 (0: an interior face).  The plan keeps B + halo below
// 8192 and at most 16 boundary conditions.
__host__ __device__ __forceinline__ unsigned pack_meta(int la, int lb, int bc) {
    return (unsigned) la | ((unsigned) lb << 13) | ((unsigned) (bc + 1) << 26);
}
inline std::vector<unsigned> packed_meta(const TilePlan& P) {
    std::vector<unsigned> w(P.meta.size() / 4);
    for (size_t i = 0; i < w.size(); i++) w[i] = pack_meta(P.meta[4 * i], P.meta[4 * i + 1], P.meta[4 * i + 2]);
    return w;
}
__device__ __forceinline__ int meta_la(unsigned w) { return (int) (w & 0x1FFFu); }
__device__ __forceinline__ int meta_lb(unsigned w) { return (int) ((w >> 13) & 0x1FFFu); }
__device__ __forceinline__ int meta_bc(unsigned w) { return (int) (w >> 26) - 1; }

// A local cell index of a tile: one of its nb cells, or one of its nh halo cells (B..).
__device__ __forceinline__ bool local_ok(int l, int nb, int B, int nh) {
    return (l >= 0 && l < nb) || (l >= B && l < B + nh);
}
// A face entry's metadata: both cells local to the tile, the boundary condition in the table.
__device__ __forceinline__ bool entry_ok(unsigned w, int nb, int B, int nh, unsigned int* err) {
    return index_ok(local_ok(meta_la(w), nb, B, nh) && local_ok(meta_lb(w), nb, B, nh) && meta_bc(w) < MAXBC, err);
}

// Cells, face entries and halo of tile t (single mesh) or of active tile t (arena).
template <bool ARENA, class T>
__device__ __forceinline__ void tile_info(const TileArgs<T>& a, int t, int& base, int& nb, int& f0, int& nf,
                                          int& h0, int& nh, int& inst) {
    if constexpr (ARENA) {
        const int4 d0 = __ldg(a.tiles + 2 * t), d1 = __ldg(a.tiles + 2 * t + 1);
        base = d0.x; nb = a.B; f0 = d0.y; nf = d0.z; inst = d0.w; h0 = d1.x; nh = d1.y;
    } else {
        base = t * a.B; nb = min(a.B, a.s.Nc - base);
        f0 = __ldg(a.foff + t); nf = __ldg(a.foff + t + 1) - f0;
        h0 = __ldg(a.hoff + t); nh = __ldg(a.hoff + t + 1) - h0;
        inst = 0;
    }
}

// What the compute warps need of a tile besides its data, written by the producer into the
// stage header with the tile's copies (published by the same mbarrier), so that the compute
// warps start a tile without dependent global loads: its descriptor, and for its instance
// the step count (limiter freezing), the dt or CFL number and the dt minimum of this step.
struct StageInfo {
    int base, nb, f0, nf, h0, nh, inst, next_inst;   // next_inst (pass 1, arena): of this CTA's next tile, -1 at the end
    double dt_or_cfl;
    double dtmin;
    long long steps;
    int t;                                            // the tile, or -1: the CTA has no more tiles
    int pad2;
};
static_assert(sizeof(StageInfo) == 64, "stage info is 64 bytes");
// Header of a CTA's shared memory: full[2] and empty[2] mbarriers (bytes 0-31), the abort
// words (32-39), then StageInfo per stage (two, from byte 64).
constexpr int kHeader = 256;
constexpr unsigned kDrainPolls = 1u << 24;

// ---------------------------------------------------------------------------------------
// PTX helpers (sm_90+ bulk copies and mbarriers; sm_80+ cp.async)

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// 1-D bulk copy global -> shared (no tensor map, no multicast); dst, src 16-B aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
// Bounded wait for an mbarrier phase.  Gives up after `polls` polls, or early once another
// thread of the CTA has given up (its abort word is set); on giving up it records the failure
// in the kernel's error word (the host reports HCFD_ETIMEOUT) and in the abort word, and
// returns false.  A thread whose wait failed never reads the stage it waited for: the
// producer then stops issuing copies, and the consumers leave their tile loop (see
// producer_loop and HCFD_TILE_LOOP_BEGIN).
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, unsigned polls, unsigned int* err,
                                          volatile int* abort) {
#pragma unroll 1
    for (unsigned i = 0; i < polls; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 255u) == 255u && *abort) return false;
    }
    atomicOr(err, 1u);
    *abort = 1;
    return false;
}
// Bounded wait for copies already issued (they only read valid global memory, so they land);
// used before a CTA exits so that nothing is written into its shared memory afterwards.
__device__ __forceinline__ void mbar_drain(unsigned long long* bar, unsigned parity, unsigned int* err) {
#pragma unroll 1
    for (unsigned i = 0; i < kDrainPolls; i++)
        if (mbar_try_wait(bar, parity)) return;
    atomicOr(err, 2u);
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ volatile int* abort_word(unsigned char* smem) { return reinterpret_cast<volatile int*>(smem + 32); }
// Set by compute threads only, before the compute barrier that follows the stage wait
// (pass 2): read after that barrier, every compute warp sees the same value.
__device__ __forceinline__ volatile int* compute_abort_word(unsigned char* smem) {
    return reinterpret_cast<volatile int*>(smem + 36);
}

// Shared-memory loads (plain loads: the __ldg helpers of hcfd_kernels.cuh are global-only).
// (chunk-plane layout of hcfd_kernels.cuh, plane stride ps = staged cell count)
__device__ __forceinline__ void lds_cell(const Cell4<double>* p, int ps, int i, double u[4]) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = q[i], b = q[ps + i];
    u[0] = a.x; u[1] = a.y; u[2] = b.x; u[3] = b.y;
}
__device__ __forceinline__ void lds_cell(const Cell4<float>* p, int, int i, float u[4]) {
    const float4 a = reinterpret_cast<const float4*>(p)[i];
    u[0] = a.x; u[1] = a.y; u[2] = a.z; u[3] = a.w;
}
__device__ __forceinline__ void lds_grad(const Grad8<double>* p, int ps, int i, double g[8]) {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int k = 0; k < 4; k++) { const double2 a = q[k * ps + i]; g[2 * k] = a.x; g[2 * k + 1] = a.y; }
}
__device__ __forceinline__ void lds_grad(const Grad8<float>* p, int ps, int i, float g[8]) {
    const float4* q = reinterpret_cast<const float4*>(p);
    const float4 a = q[i], b = q[ps + i];
    g[0] = a.x; g[1] = a.y; g[2] = a.z; g[3] = a.w; g[4] = b.x; g[5] = b.y; g[6] = b.z; g[7] = b.w;
}
// Face records of a tile are stored pair-major: four planes of pairs, (nx, ny), (Af, If),
// (rLx, rLy), (rRx, rRy); pair j of entry e at index j nf + e of the pair array (16 bytes a pair
// in double, 8 in float).  One load brings a pair, and consecutive threads reading consecutive
// entries touch consecutive words (no bank conflicts).
template <class T> struct PairOf;
template <> struct PairOf<double> { using type = double2; };
template <> struct PairOf<float> { using type = float2; };
template <class T>
__device__ __forceinline__ typename PairOf<T>::type ldp(const T* p, int nf, int j, int e) {
    return reinterpret_cast<const typename PairOf<T>::type*>(p)[j * nf + e];
}
template <class T>
__device__ __forceinline__ void stp(T* p, int nf, int j, int e, T x, T y) {
    typename PairOf<T>::type v;
    v.x = x; v.y = y;
    reinterpret_cast<typename PairOf<T>::type*>(p)[j * nf + e] = v;
}
// Records of 8 values (pass 1, and pass 2 when it shares pass 1's plan, the arena's too):
// pairs (nx, ny), (Af, If), (rLx, rLy), (rRx, rRy).  Records of 7 values (pass 2 on a plan of
// its own, which never reads If): pairs (nx, ny), (rLx, rLy), (rRx, rRy), then Af alone in a
// plane of scalars.  rplane gives the pair plane of rL (rR follows it).
__device__ __forceinline__ int rplane(int rec) { return rec == 7 ? 1 : 2; }
template <class T>
__device__ __forceinline__ T lds_area(const T* p, int nf, int e, int rec) {
    return rec == 7 ? p[6 * nf + e] : p[2 * (nf + e)];
}

template <class T>
__device__ __forceinline__ void lds_geo(const T* p, int nf, int e, FaceGeo<T>& g) {
    const auto a = ldp(p, nf, 0, e), b = ldp(p, nf, 1, e), c = ldp(p, nf, 2, e), d = ldp(p, nf, 3, e);
    g.nx = a.x; g.ny = a.y; g.Af = b.x; g.If = b.y; g.rLx = c.x; g.rLy = c.y; g.rRx = d.x; g.rRy = d.y;
}

// Normal, length and interpolation weight (pass 1 reads the r vector of one side apart).
template <class T>
__device__ __forceinline__ void lds_geo4(const T* p, int nf, int e, FaceGeo<T>& g) {
    const auto a = ldp(p, nf, 0, e), b = ldp(p, nf, 1, e);
    g.nx = a.x; g.ny = a.y; g.Af = b.x; g.If = b.y;
}

// Normal and length only (the components pass 2's flux write leaves intact).
template <class T>
__device__ __forceinline__ void lds_geo3(const T* p, int nf, int e, int rec, T& nx, T& ny, T& Af) {
    const auto a = ldp(p, nf, 0, e);
    nx = a.x; ny = a.y; Af = lds_area(p, nf, e, rec);
}

__host__ __device__ constexpr size_t align128(size_t x) { return (x + 127) & ~size_t(127); }

// Shared-memory layout of one CTA: two mbarriers and two staging buffers (double buffering:
// tile i+1 is in flight while tile i is computed).  One staging buffer holds the tile's and
// its halo's cells (and limited gradients in pass 2), its face records and metadata, its
// slot table and its iv.  Pass 2 keeps its fluxes in the staged face records, so a CTA
// needs no other scratch (three CTAs of 128 + 32 threads fit an SM at 128-cell tiles).
template <class T>
struct TileSmem {
    size_t u, g, geo, meta, cslot, iv, stage, total;   // byte offsets within a stage
    __host__ __device__ TileSmem(int B, int Hmax, int Fmax, int W, int Wp, bool pass2) {
        size_t p = 0;
        u = p;     p += align128((size_t) (B + Hmax) * sizeof(Cell4<T>));
        g = p;     if (pass2) p += align128((size_t) (B + Hmax) * sizeof(Grad8<T>));
        geo = p;   p += align128((size_t) Fmax * sizeof(FaceGeo<T>));
        meta = p;  p += align128((size_t) Fmax * 4);
        cslot = p; p += align128((size_t) B * Wp * sizeof(short));
        iv = p;    p += align128((size_t) B * sizeof(T));
        stage = p;
        total = kHeader + 2 * stage;
        (void) W;
    }
};

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Arrival on `bar` once all cp.async operations issued so far by this thread have landed;
// counts as one of the barrier's expected arrivals (.noinc).
__device__ __forceinline__ void cp_async_arrive_noinc(unsigned long long* bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Barrier over the compute warps only (named barrier 1; the producer warp never joins it).
__device__ __forceinline__ void compute_sync(int nthreads) {
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

// Producer warp: for each of this CTA's tiles, waits until the compute warps have released
// the staging buffer, then lane 0 arms the buffer's `full` mbarrier with the byte count of
// the bulk copies and issues them, and every lane gathers its share of the halo cells with
// cp.async and signals their completion on the same mbarrier.  The `full` barrier therefore
// completes when all of the tile's data has landed: 1 expect-tx arrival + 32 cp.async
// arrivals + the transaction bytes.
// Once any wait of the CTA has given up, the producer issues nothing more; before it
// returns it waits for the copies it has issued (the last armed phase of each buffer; earlier
// ones completed before their buffer was re-armed), so no copy lands after the CTA exits.
// Tile queue: lane 0 of the producer warp issues the claim of a tile at the top of an
// iteration (claim_issue) and the warp takes its result at the end (claim_take), so that the
// atomic's round trip overlaps the iteration's staging.
template <class T>
__device__ __forceinline__ int claim_issue(const TileArgs<T>& a, int lane) {
    return (a.claim && lane == 0) ? atomicAdd(a.claim, 1) : 0;
}
template <class T>
__device__ __forceinline__ int claim_take(const TileArgs<T>& a, int t, int pending) {
    if (!a.claim) return t + (int) gridDim.x;
    return (int) gridDim.x + __shfl_sync(0xffffffffu, pending, 0);
}

template <class T, bool PASS2, bool ARENA>
__device__ __forceinline__ void producer_loop(const TileArgs<T>& a, unsigned char* smem, unsigned long long* full,
                                              unsigned long long* empty, const TileSmem<T>& L) {
    const int lane = threadIdx.x & 31;
    constexpr int CU = sizeof(Cell4<T>) / 16, CG = PASS2 ? sizeof(Grad8<T>) / 16 : 0;
    const int NL = a.B + a.Hmax;   // plane stride of the staged cells
    volatile int* abort = abort_word(smem);
    int armed[2] = {-1, -1};       // last iteration whose copies were issued into each buffer
    unsigned iter = 0;
    // the current tile t and the next tn are known at the top of an iteration; the tile after
    // tn is claimed during the iteration
    int t = blockIdx.x;
    int tn = claim_take(a, t, claim_issue(a, lane));
    int pending = 0;
    for (;; iter++, t = tn, tn = t < a.ntiles ? claim_take(a, t, pending) : t) {
        const int buf = iter & 1;
        if (tn < a.ntiles) pending = claim_issue(a, lane);
        if (__any_sync(0xffffffffu, *abort)) break;
        if (t >= a.ntiles) {
            // no more tiles: a stage with tile -1 and nothing copied ends the compute warps' loop
            if (iter >= 2 && !__all_sync(0xffffffffu, mbar_wait(empty + buf, ((iter >> 1) - 1) & 1, a.polls, a.err, abort)))
                break;
            if (lane == 0) {
                reinterpret_cast<StageInfo*>(smem + 64)[buf].t = -1;
                mbar_arrive_expect_tx(full + buf, 0u);
            }
            cp_async_arrive_noinc(full + buf);
            armed[buf] = (int) iter;
            break;
        }
        // the tile's descriptor and its instance's scalars are loaded before the wait for the
        // stage, so that their latency hides behind it (none of them changes during the kernel
        // in a way the kernel reads: dt minima and step counts come from earlier kernels)
        int base, nb, f0, nf, h0, nh, inst;
        tile_info<ARENA>(a, t, base, nb, f0, nf, h0, nh, inst);
        double v_dt = 0.0, v_dtmin = 0.0;
        long long v_steps = 0;
        int v_next = -1;
        if (lane == 0) {
            if constexpr (ARENA) {
                v_dt = __ldg(a.inst_dt + inst);
                v_dtmin = __longlong_as_double((long long) a.inst_dtmin[2 * inst + a.par]);
                v_steps = a.inst_stats[inst].steps;
                if (!PASS2 && tn < a.ntiles) v_next = __ldg(&a.tiles[2 * tn].w);
            } else {
                v_dt = a.s.dt_or_cfl;
                v_dtmin = __longlong_as_double((long long) *a.s.dtmin);
                v_steps = a.s.stats->steps;
            }
        }
        if (iter >= 2 && !__all_sync(0xffffffffu, mbar_wait(empty + buf, ((iter >> 1) - 1) & 1, a.polls, a.err, abort)))
            break;
        if (t == a.skip_tile) continue;      // failure injection: nothing armed, nothing in flight
        bool good = true;
        if constexpr (kChecked) {
            // a descriptor outside the arrays or the staging capacity: the tile is staged empty
            good = index_ok(base >= 0 && nb >= 0 && nb <= a.B && base + nb <= a.ps && base + a.B <= a.ncap &&
                            f0 >= 0 && nf >= 0 && nf <= a.Fmax && f0 + nf <= a.nentries &&
                            h0 >= 0 && nh >= 0 && nh <= a.Hmax && h0 + nh <= a.nhalo, a.err);
            if (!good) nb = nf = nh = 0;
        }
        unsigned char* st = smem + kHeader + buf * L.stage;
        Cell4<T>* sU = reinterpret_cast<Cell4<T>*>(st + L.u);
        Grad8<T>* sG = reinterpret_cast<Grad8<T>*>(st + L.g);
        if (lane == 0) {
            const unsigned bu = nb * sizeof(Cell4<T>), bg = PASS2 ? nb * sizeof(Grad8<T>) : 0u;
            const unsigned bf = nf * a.rec * (unsigned) sizeof(T), bm = nf * 4u;
            const unsigned bs = a.B * a.Wp * sizeof(short), bi = a.B * sizeof(T);
            // the tile's descriptor and instance scalars, published by the release of the
            // arrive below
            StageInfo* si = reinterpret_cast<StageInfo*>(smem + 64) + buf;
            si->base = base; si->nb = nb; si->f0 = f0; si->nf = nf; si->h0 = h0; si->nh = nh; si->inst = inst;
            si->t = t;
            si->next_inst = v_next;                  // pass 1 in arena mode only
            si->dt_or_cfl = v_dt;
            si->dtmin = v_dtmin;
            si->steps = v_steps;
            if (!good) {
                mbar_arrive_expect_tx(full + buf, 0u);   // nothing copied (checked build)
            } else {
            mbar_arrive_expect_tx(full + buf, bu + bg + bf + bm + bs + bi);
            // one bulk copy per 16-byte chunk plane of the tile's cell range
#pragma unroll
            for (int j = 0; j < CU; j++)
                bulk_g2s(reinterpret_cast<char*>(sU) + (size_t) 16 * j * NL,
                         reinterpret_cast<const char*>(a.s.U) + 16 * ((size_t) j * a.ps + base), nb * 16u, full + buf);
            if (PASS2) {
#pragma unroll
                for (int j = 0; j < CG; j++)
                    bulk_g2s(reinterpret_cast<char*>(sG) + (size_t) 16 * j * NL,
                             reinterpret_cast<const char*>(a.s.phiG) + 16 * ((size_t) j * a.ps + base), nb * 16u,
                             full + buf);
            }
            if (bf) {
                bulk_g2s(st + L.geo, a.tgeo + (size_t) f0 * a.rec, bf, full + buf);
                bulk_g2s(st + L.meta, a.tmeta + f0, bm, full + buf);
            }
            bulk_g2s(st + L.cslot, a.cslot + (size_t) base * a.Wp, bs, full + buf);
            bulk_g2s(st + L.iv, a.s.iv + base, bi, full + buf);
            }
        }
        for (int h = lane; h < nh; h += 32) {
            const int ci = __ldg(a.halo + h0 + h);
            if (!index_ok(ci >= 0 && ci < a.ps, a.err)) continue;
#pragma unroll
            for (int j = 0; j < CU; j++)
                cp_async16(reinterpret_cast<char*>(sU) + 16 * ((size_t) j * NL + a.B + h),
                           reinterpret_cast<const char*>(a.s.U) + 16 * ((size_t) j * a.ps + ci));
#pragma unroll
            for (int j = 0; j < CG; j++)
                cp_async16(reinterpret_cast<char*>(sG) + 16 * ((size_t) j * NL + a.B + h),
                           reinterpret_cast<const char*>(a.s.phiG) + 16 * ((size_t) j * a.ps + ci));
        }
        cp_async_arrive_noinc(full + buf);
        armed[buf] = (int) iter;
    }
    cp_async_wait_all();
    for (int b = 0; b < 2; b++)
        if (armed[b] >= 0) mbar_drain(full + b, ((unsigned) armed[b] >> 1) & 1, a.err);
}

// Residual / non-finite / dt bookkeeping shared by the last pass of a step.
template <class T>
__device__ __forceinline__ void finish_step(const StepArgs<T>& a, double r2, int bad, double dt_used) {
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
            if (a.time_mode != TM_FIXED) *a.dtmin_next = 0x7FF0000000000000ULL;
        }
    }
}

// ---------------------------------------------------------------------------------------

__device__ __forceinline__ void lds_slots(const short* p, int Wp, short cs[8]) {
    if (Wp == 3) {
        cs[0] = p[0]; cs[1] = p[1]; cs[2] = p[2];
        cs[3] = cs[4] = cs[5] = cs[6] = cs[7] = -1;
    } else if (Wp == 4) {
        const short4 a = *reinterpret_cast<const short4*>(p);
        cs[0] = a.x; cs[1] = a.y; cs[2] = a.z; cs[3] = a.w;
        cs[4] = cs[5] = cs[6] = cs[7] = -1;
    } else {
        const int4 a = *reinterpret_cast<const int4*>(p);
        const short* q = reinterpret_cast<const short*>(&a);
#pragma unroll
        for (int k = 0; k < 8; k++) cs[k] = q[k];
    }
}

// One face entry of pass 2: operands gathered from shared memory and reduced at once to the
// MUSCL states on both sides (Flux.cpp:83-87), then the Rusanov flux in the face's own
// L -> R orientation.  Only the reconstructed states stay live between load and flux.
template <class T>
struct FaceIn {
    T uoL[4], uqR[4], nx, ny, Af;
    int e;
    __device__ __forceinline__ void load(const Cell4<T>* sU, const Grad8<T>* sG, int NL, const T* sGeo,
                                         const unsigned* sMeta, int nf, int rec, int e_) {
        e = e_;
        const unsigned w = sMeta[e];
        const int bc = meta_bc(w);
        const int mx = meta_la(w), my = meta_lb(w);
        const int rp = rplane(rec);
        FaceGeo<T> g;
        {
            const auto n2 = ldp(sGeo, nf, 0, e), rl = ldp(sGeo, nf, rp, e), rr = ldp(sGeo, nf, rp + 1, e);
            g.nx = n2.x; g.ny = n2.y; g.rLx = rl.x; g.rLy = rl.y; g.rRx = rr.x; g.rRy = rr.y;
        }
        nx = g.nx; ny = g.ny; Af = lds_area(sGeo, nf, e, rec);
        T uL[4], uR[4], gL[8];
        lds_cell(sU, NL, mx, uL);
        lds_cell(sU, NL, my, uR);
        lds_grad(sG, NL, mx, gL);
        if (bc >= 0) {
            // Ghost on the right: -grad and the same phi as the interior cell with r_R = -r_L
            // (BoundaryConditions/Base.cpp:29-53, Domain.cpp:84-88): the same increment.
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const T du = gL[2 * v] * g.rLx + gL[2 * v + 1] * g.rLy;
                uoL[v] = uL[v] + du;
                uqR[v] = uR[v] + du;
            }
        } else {
            T gR[8];
            lds_grad(sG, NL, my, gR);
#pragma unroll
            for (int v = 0; v < 4; v++) {
                uoL[v] = uL[v] + (gL[2 * v] * g.rLx + gL[2 * v + 1] * g.rLy);
                uqR[v] = uR[v] + (gR[2 * v] * g.rRx + gR[2 * v + 1] * g.rRy);
            }
        }
    }
    __device__ __forceinline__ void flux(T gma, T F[4]) const { rusanov(uoL, uqR, nx, ny, gma, F); }
    // F over the two r pairs of this entry's staged record: only this thread reads them in
    // pass 2, and it has read them already.  With AF the product A_f F is stored instead (the
    // compensated FP32 sums round that product before adding it, so forming it once per face
    // gives the same bits as forming it in each of the two cells).
    template <bool AF>
    __device__ __forceinline__ void store(T* sGeo, int nf, int rec, const T F[4]) const {
        const int rp = rplane(rec);
        if (AF) {
            stp(sGeo, nf, rp, e, F[0] * Af, F[1] * Af);
            stp(sGeo, nf, rp + 1, e, F[2] * Af, F[3] * Af);
        } else {
            stp(sGeo, nf, rp, e, F[0], F[1]);
            stp(sGeo, nf, rp + 1, e, F[2], F[3]);
        }
    }
};

// Warp-specialised persistent tile loop.  The last warp of the CTA is the producer
// (producer_loop); the first NT = blockDim.x - 32 threads compute.  Compute iteration i
// reads staging buffer i & 1 once its `full` barrier completes and releases it on its
// `empty` barrier (one arrival per compute warp) when done.  The tile comes with the stage
// (StageInfo::t); after the CTA's last tile the producer stages tile -1 with nothing copied,
// and the compute warps leave the loop on it (in pass 2 after the face-phase barrier, which
// every compute warp meets once more).
// A compute warp whose stage wait gives up reads nothing of that stage.  In pass 1 (no
// barrier among the compute warps inside the loop) it leaves the loop at once.  In pass 2
// it marks the compute abort word and skips the face phase (`staged` false); every compute
// warp then meets at the compute barrier that ends the face phase and leaves the loop
// there if any of them gave up, so none is left waiting at that barrier.
#define HCFD_TILE_LOOP_BEGIN(PASS2, ARENA)                                                       \
    const int NT = blockDim.x - 32;                                                              \
    const int NL = a.B + a.Hmax;                                                                 \
    unsigned long long* full = reinterpret_cast<unsigned long long*>(smem);                      \
    unsigned long long* empty = full + 2;                                                        \
    if (threadIdx.x == 0) {                                                                      \
        mbar_init(full, 33); mbar_init(full + 1, 33);                                            \
        mbar_init(empty, NT / 32); mbar_init(empty + 1, NT / 32);                                \
        *abort_word(smem) = 0;                                                                   \
        *compute_abort_word(smem) = 0;                                                           \
        fence_mbar_init();                                                                       \
    }                                                                                            \
    __syncthreads();                                                                             \
    if ((int) threadIdx.x >= NT) {                                                               \
        producer_loop<T, PASS2, ARENA>(a, smem, full, empty, L);                                 \
    } else {                                                                                     \
    if (a.claim_reset && blockIdx.x == 0 && threadIdx.x == 0) *a.claim_reset = 0;               \
    for (unsigned iter = 0;; iter++) {                                                           \
        const int buf = iter & 1;                                                                \
        unsigned char* st = smem + kHeader + buf * L.stage;                                      \
        const bool staged = __all_sync(0xffffffffu,                                              \
                                       mbar_wait(full + buf, (iter >> 1) & 1, a.polls, a.err,    \
                                                 abort_word(smem)));                             \
        if (!PASS2 && !staged) break;                                                            \
        if (PASS2 && !staged && (threadIdx.x & 31) == 0) *compute_abort_word(smem) = 1;          \
        const StageInfo& si = reinterpret_cast<const StageInfo*>(smem + 64)[buf];                \
        const int t = staged ? si.t : 0;                                                         \
        const bool fin = staged && t < 0;     /* the producer has no more tiles */               \
        if (!PASS2 && fin) break;                                                                \
        const int base = si.base, nb = si.nb, h0t = si.h0, inst = si.inst;                      \
        const Cell4<T>* sU = reinterpret_cast<const Cell4<T>*>(st + L.u);                        \
        const T* sGeo = reinterpret_cast<const T*>(st + L.geo);                                  \
        const int nfl = si.nf;                                                                   \
        const unsigned* sMeta = reinterpret_cast<const unsigned*>(st + L.meta);                  \
        const short* sSlot = reinterpret_cast<const short*>(st + L.cslot);                       \
        const T* sIv = reinterpret_cast<const T*>(st + L.iv);

#define HCFD_TILE_LOOP_END                                                                       \
        __syncwarp();                                                                            \
        if ((threadIdx.x & 31) == 0) mbar_arrive(empty + buf);                                   \
    }                                                                                            \
    }

template <class T, int W, bool ARENA>
__global__ void __launch_bounds__(288) tile_pass1_kernel(const TileArgs<T> a) {
    extern __shared__ __align__(128) unsigned char smem[];
    const TileSmem<T> L(a.B, a.Hmax, a.Fmax, W, a.Wp, false);
    const StepArgs<T>& s = a.s;
    T xmx = T(0);                        // largest iv * lam (see dt_of_max)
    HCFD_TILE_LOOP_BEGIN(false, ARENA)
    const int lmode = limiter_mode(si.steps, s.freeze_after);
    for (int c = threadIdx.x; c < nb; c += NT) {
        short cs[8];
        lds_slots(sSlot + c * a.Wp, a.Wp, cs);
        if (cs[0] < 0) continue;
        T u[4];
        lds_cell(sU, NL, c, u);
        const T iv = sIv[c];
        T G[4][2], umin[4], umax[4], ro[W][2];
#pragma unroll
        for (int v = 0; v < 4; v++) { G[v][0] = T(0); G[v][1] = T(0); umin[v] = u[v]; umax[v] = u[v]; }
        T cu = T(0), cv = T(0), ca = T(0), lam = T(0);
        if (s.time_mode != TM_FIXED) cell_speed(u, s.gma, cu, cv, ca);
#pragma unroll
        for (int k = 0; k < W; k++) {
            ro[k][0] = T(0); ro[k][1] = T(0);
            if (cs[k] < 0) continue;
            int e = cs[k] >> 1;
            const bool isL = (cs[k] & 1) == 0;
            if constexpr (kChecked)    // a bad index is replaced by entry 0 / tile cell 0 (no branch)
                e = index_ok(e < nfl, a.err) ? e : 0;
            FaceGeo<T> g;
            lds_geo4(sGeo, nfl, e, g);
            int nbl = isL ? meta_lb(sMeta[e]) : meta_la(sMeta[e]);
            if constexpr (kChecked)
                nbl = index_ok(local_ok(nbl, nb, a.B, si.nh), a.err) ? nbl : 0;
            T un[4];
            lds_cell(sU, NL, nbl, un);
            // GaussGreen.cpp:25-28: uf = u_CL If + u_CR (1 - If), added into CL and taken from
            // CR.  The side is folded into two weights and a signed length once per face
            // (face_weights) instead of selecting four left/right states and branching per
            // variable.
            T ws, wn, sA;
            face_weights(isL, g.If, g.Af, ws, wn, sA);
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const T uf = u[v] * ws + un[v] * wn;
                const T tt = uf * sA;
                G[v][0] += tt * g.nx;
                G[v][1] += tt * g.ny;
                umin[v] = fmin(umin[v], un[v]);                  // Limiter.cpp:31-39
                umax[v] = fmax(umax[v], un[v]);
            }
            // this cell's own centre-to-face vector: one pair, at its side's plane
            const auto rr = ldp(sGeo, nfl, isL ? 2 : 3, e);
            ro[k][0] = rr.x;
            ro[k][1] = rr.y;
            if (s.time_mode != TM_FIXED) lam += wave(cu, cv, ca, g);
        }
        T e2 = T(0);
        if (s.limiter == LIM_VENKAT) {
            const T kh = s.venkat_K * qsqrt(qrcp(iv));
            e2 = kh * kh * kh;
        }
        const T eps = T(1e-9);
        T out[8], phis[4];
        if (lmode == LIM_FROZEN) ld_cell(s.phiF, a.ps, base + c, phis);
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const T gx = G[v][0] * iv, gy = G[v][1] * iv;
            T phi = T(1);
            if (lmode == LIM_FROZEN) {
                phi = phis[v];
            } else {
#pragma unroll
                for (int k = 0; k < W; k++) {
                    if (cs[k] < 0) continue;
                    const T d = gx * ro[k][0] + gy * ro[k][1];
                    T pf = T(1);                                     // Limiter.cpp:67-71
                    if (d > eps || d < -eps)
                        pf = face_limiter(s.limiter, (d > eps) ? umax[v] - u[v] : umin[v] - u[v], d, e2);
                    phi = fmin(phi, pf);
                }
            }
            phis[v] = phi;
            out[2 * v] = phi * gx;
            out[2 * v + 1] = phi * gy;
        }
        if (lmode == LIM_RECORD) st_cell(s.phiF, a.ps, base + c, phis);
        st_grad(s.phiG, a.ps, base + c, out);
        if (s.time_mode != TM_FIXED) xmx = fmax(xmx, iv * lam);
    }
    if constexpr (ARENA) {
        // per-instance minimum (exact and order-free): each warp carries its minimum across
        // this CTA's consecutive tiles of one instance and posts it with one atomic when the
        // next tile belongs to another instance, so a large instance sees a few atomics per
        // CTA rather than one per warp and tile on a single address
        if (s.time_mode != TM_FIXED) {
            if (si.next_inst != inst) {
                const double m = dt_of_max(warp_max(xmx));
                if ((threadIdx.x & 31) == 0 && m < 1e300)
                    atomicMin(a.inst_dtmin + 2 * inst + a.par, (unsigned long long) __double_as_longlong(m));
                xmx = T(0);
            }
        }
    }
    HCFD_TILE_LOOP_END
    if (!ARENA && s.time_mode != TM_FIXED) {
        __shared__ T sm[32];
        T m = warp_max(xmx);
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if (lane == 0) sm[wid] = m;
        __syncthreads();
        if (wid == 0) {
            m = lane < (int) (blockDim.x >> 5) ? sm[lane] : T(0);
            const double d = dt_of_max(warp_max(m));
            if (lane == 0 && d < 1e300) atomicMin(s.dtmin, (unsigned long long) __double_as_longlong(d));
        }
    }
}

template <class T, int W, bool COMP, bool ARENA>
__global__ void __maxnreg__(128) tile_pass2_kernel(const TileArgs<T> a) {
    extern __shared__ __align__(128) unsigned char smem[];
    const TileSmem<T> L(a.B, a.Hmax, a.Fmax, W, a.Wp, true);
    const StepArgs<T>& s = a.s;
    double dt_used = 0.0;
    double r2 = 0.0;
    int bad = 0;
    HCFD_TILE_LOOP_BEGIN(true, ARENA)
    const T cfl_or_dt = T(si.dt_or_cfl);
    if (staged && !fin) dt_used = (s.time_mode == TM_FIXED) ? si.dt_or_cfl : si.dt_or_cfl * si.dtmin;
    const Grad8<T>* sG = reinterpret_cast<const Grad8<T>*>(st + L.g);
    // a stage whose wait gave up is not read, nor the closing stage (tile -1)
    const int nf = (staged && !fin) ? nfl : 0;
    // face phase: one Rusanov flux per face entry (Flux.cpp:19-38).  Each thread takes two
    // entries per round and computes both before storing either, so the two independent
    // FP64 dependency chains (divisions, square roots) interleave.
    // Threads below nf - NT (per round) have a second entry.  In FP64, whole warps take the
    // one-entry path when none of their threads has one (the warp that straddles the boundary
    // takes the two-entry path throughout, its threads without a second entry computing theirs
    // twice, so that no warp runs both paths one after the other); this saves FP64 work.  In
    // FP32 every warp takes the two-entry path: the flux is cheap there, and measured on the
    // B200 the split costs more than it saves.
    T* sGeoW = reinterpret_cast<T*>(st + L.geo);
    for (int e = threadIdx.x; e < nf; e += 2 * NT) {
        const int base2 = e - (int) threadIdx.x;                 // first entry of this round
        const int pairs = min(NT, max(0, nf - base2 - NT));      // threads with a second entry
        if (sizeof(T) == 4 || (int) (threadIdx.x & ~31u) < pairs) {
            const int eB = (e + NT < nf) ? e + NT : e;
            if constexpr (kChecked)
                if (!entry_ok(sMeta[e], nb, a.B, si.nh, a.err) || !entry_ok(sMeta[eB], nb, a.B, si.nh, a.err)) continue;
            FaceIn<T> A, Bq;
            A.load(sU, sG, NL, sGeo, sMeta, nf, a.rec, e);
            Bq.load(sU, sG, NL, sGeo, sMeta, nf, a.rec, eB);
            T FA[4], FB[4];
            A.flux(s.gma, FA);
            Bq.flux(s.gma, FB);
            A.template store<COMP>(sGeoW, nf, a.rec, FA);
            if (eB != e) Bq.template store<COMP>(sGeoW, nf, a.rec, FB);
        } else {
            if constexpr (kChecked)
                if (!entry_ok(sMeta[e], nb, a.B, si.nh, a.err)) continue;
            FaceIn<T> A;
            A.load(sU, sG, NL, sGeo, sMeta, nf, a.rec, e);
            T FA[4];
            A.flux(s.gma, FA);
            A.template store<COMP>(sGeoW, nf, a.rec, FA);
        }
    }
    compute_sync(NT);
    // some compute warp's stage wait gave up, or the closing stage (every compute warp that
    // read the stage sees its tile -1; one whose wait gave up sees the abort word)
    if (*compute_abort_word(smem) || fin) break;
    // cell phase: slots in increasing face order, update, ghost refresh
    for (int c = threadIdx.x; c < nb; c += NT) {
        short cs[8];
        lds_slots(sSlot + c * a.Wp, a.Wp, cs);
        if (cs[0] < 0) continue;
        T u[4];
        lds_cell(sU, NL, c, u);
        const T iv = sIv[c];
        T R[4], Rc[4];
#pragma unroll
        for (int v = 0; v < 4; v++) { R[v] = T(0); Rc[v] = T(0); }
        T cu = T(0), cv = T(0), ca = T(0), lam = T(0);
        if (s.time_mode == TM_LOCAL) cell_speed(u, s.gma, cu, cv, ca);
#pragma unroll
        for (int k = 0; k < W; k++) {
            if (cs[k] < 0) continue;
            const bool isL = (cs[k] & 1) == 0;
            int e = cs[k] >> 1;
            if constexpr (kChecked)
                e = index_ok(e < nf, a.err) ? e : 0;
            const int rp = rplane(a.rec);
            const auto F01 = ldp(sGeo, nf, rp, e), F23 = ldp(sGeo, nf, rp + 1, e);
            const T Fk[4] = {F01.x, F01.y, F23.x, F23.y};
            T Af = T(0);
            if constexpr (!COMP) Af = lds_area(sGeo, nf, e, a.rec);
#pragma unroll
            for (int v = 0; v < 4; v++) {                        // Flux.cpp:39-42
                const T Fv = Fk[v];
                if constexpr (COMP) {                            // Fv holds A_f F here
                    two_sum(R[v], Rc[v], isL ? -Fv : Fv);
                } else {
                    if (isL) R[v] -= Af * Fv;
                    else     R[v] += Af * Fv;
                }
            }
            if (s.time_mode == TM_LOCAL) {                       // the normal only for the local dt
                FaceGeo<T> g;
                lds_geo3(sGeo, nf, e, a.rec, g.nx, g.ny, g.Af);
                lam += wave(cu, cv, ca, g);
            }
        }
        T dt;
        if (s.time_mode == TM_LOCAL) dt = cfl_or_dt * qrcp(iv * lam);
        else dt = T(dt_used);
        T un_[4];
#pragma unroll
        for (int v = 0; v < 4; v++) {
            T Rv = COMP ? R[v] + Rc[v] : R[v];
            Rv = Rv * iv;                                        // Flux.cpp:45-49
            un_[v] = u[v] + dt * Rv;                             // Euler.cpp:107-113
            if (v == 0) r2 += (double) Rv * (double) Rv;
            bad |= !isfinite(un_[v]);
        }
        st_cell(s.Unew, a.ps, base + c, un_);
        // ghost refresh (Euler.cpp:96, :138-142): this cell is its ghosts' only neighbour
#pragma unroll
        for (int k = 0; k < W; k++) {
            if (cs[k] < 0 || (cs[k] & 1)) continue;
            const int e = cs[k] >> 1;
            const unsigned w = sMeta[e];
            const int bc = meta_bc(w);
            if (bc < 0) continue;
            const int lb = meta_lb(w);
            if (!index_ok(local_ok(lb, nb, a.B, si.nh) && bc < MAXBC, a.err)) continue;
            const int gi = lb < a.B ? base + lb : __ldg(a.halo + h0t + lb - a.B);
            if (!index_ok(gi >= 0 && gi < a.ps, a.err)) continue;
            T gnx, gny, gA;
            lds_geo3(sGeo, nf, e, a.rec, gnx, gny, gA);
            T ug[4];
            const BCTable* bt = ARENA ? a.inst_bc + inst : &s.bc;
            ghost_state(bt->type[bc], un_, gnx, gny, s.gma, bt->UBC[bc], bt->QBC[bc], ug);
            st_cell(s.Unew, a.ps, gi, ug);
        }
    }
    if constexpr (ARENA) {
        // per-tile residual: one partial per warp (fixed order, no barrier); the finalize
        // kernel sums an instance's partials in order
        const double w = warp_sum(r2);
        const int wb = __any_sync(0xffffffffu, bad);
        if ((threadIdx.x & 31) == 0) {
            const int k = t * (NT >> 5) + (int) (threadIdx.x >> 5);
            a.tile_r2[k] = w;
            a.tile_bad[k] = wb;
        }
        r2 = 0.0;
        bad = 0;
    }
    HCFD_TILE_LOOP_END
    if constexpr (!ARENA) finish_step(s, r2, bad, dt_used);
}

// Face records in tile order, pair-major per tile, rec values each (8 or 7; see rplane):
// tile t with entries [f0, f0 + nf) starts at tgeo[rec f0] (zeros for padding).
template <class T>
__global__ void gather_geo_kernel(int ntiles, const int* __restrict__ foff, const int* __restrict__ efid,
                                  const FaceGeo<double>* __restrict__ geo, T* __restrict__ tgeo, int rec) {
    const int t = blockIdx.x;
    if (t >= ntiles) return;
    const int f0 = foff[t], nf = foff[t + 1] - f0;
    T* out = tgeo + (size_t) rec * f0;
    for (int e = threadIdx.x; e < nf; e += blockDim.x) {
        const int f = efid[f0 + e];
        double c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (f >= 0) {
            const FaceGeo<double> g = geo[f];
            c[0] = g.nx; c[1] = g.ny; c[2] = g.Af; c[3] = g.If; c[4] = g.rLx; c[5] = g.rLy; c[6] = g.rRx; c[7] = g.rRy;
        }
        if (rec == 7) {
            stp(out, nf, 0, e, T(c[0]), T(c[1]));
            stp(out, nf, 1, e, T(c[4]), T(c[5]));
            stp(out, nf, 2, e, T(c[6]), T(c[7]));
            out[6 * nf + e] = T(c[2]);
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) stp(out, nf, j, e, T(c[2 * j]), T(c[2 * j + 1]));
        }
    }
}

}  // namespace hcfd
