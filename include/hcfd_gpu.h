/* hcfd_gpu.h — C ABI of the B200 solver for the per-step residual-and-update loop of the
 * 2-D unstructured cell-centred finite-volume Euler solver of
 * Hasti-Jalal-Aldeen/CFD_Optimisations.
 *
 * Every entry point below names the reference interface it stands in for.  The reference
 * has no C ABI of its own: its solver is a set of C++ classes (includes/Base/*.hpp) built
 * into one executable, and its only historical foreign-function boundary was a ctypes
 * binding (interface/LEGACY/Run.py:98-141).  This header is what such a binding, or the
 * C++ drop-in in hcfd_gpu.hpp, calls.
 *
 * Conventions
 *  - Plain pointers and sizes, no C++ types.  Status codes: HCFD_OK (0) or a negative
 *    HCFD_E* value; hcfd_last_error() gives the text of the last failure on the calling
 *    thread.
 *  - Host arrays passed in are copied; the caller keeps ownership.  The library owns all
 *    device memory.  Each solver handle owns one CUDA stream; a handle is not thread-safe,
 *    distinct handles may be used from distinct threads.
 *  - State arrays are variable-major (4 arrays of Nc doubles: rho, rho u, rho v, E), the
 *    layout of the reference's `double* U[NVARS]` (includes/Base/TimeIntegrators.hpp:38-42).
 *  - There is no CPU fallback: without a usable CUDA device every solver call fails with
 *    HCFD_ECUDA.
 */
#ifndef HCFD_GPU_H
#define HCFD_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------- */
#define HCFD_OK           0
#define HCFD_EINVAL      -1   /* bad argument or malformed mesh                            */
#define HCFD_ENOMEM      -2   /* host or device allocation failed                          */
#define HCFD_ECUDA       -3   /* CUDA runtime error (no device, launch failure, ...)       */
#define HCFD_ENONFINITE  -4   /* a NaN or Inf appeared in the state                        */
#define HCFD_ETIMEOUT    -5   /* a bounded device wait gave up                             */
#define HCFD_EIO         -6   /* file could not be read or written                         */
#define HCFD_EAGAIN      -7   /* arena full: retry after a retirement                      */

/* Boundary-condition types, same values as Base::BCtype
 * (includes/Base/BoundaryConditions.hpp:6-13). */
enum hcfd_bctype {
    HCFD_SYMMETRY = 0, HCFD_WALL = 1, HCFD_SUPINLET = 2,
    HCFD_SUBINLET = 3, HCFD_SUPOUTLET = 4, HCFD_SUBOUTLET = 5
};

/* Limiter: Barth-Jespersen (the reference's Limiter::limit_gradient,
 * src/Base/Limiter.cpp:19-77) or Venkatakrishnan with constant K (not in the reference). */
enum hcfd_limiter { HCFD_LIMITER_BJ = 0, HCFD_LIMITER_VENKAT = 1 };

/* How a step picks dt.  HCFD_FIXED_DT is the reference's only mode (Euler::run(T, dt,
 * dt_out), src/Base/Euler.cpp:79-105).  The CFL modes are not in the reference. */
enum hcfd_time_mode { HCFD_FIXED_DT = 0, HCFD_GLOBAL_CFL = 1, HCFD_LOCAL_CFL = 2 };

/* Arithmetic of the step.  HCFD_FP64 follows the reference's double arithmetic.
 * HCFD_FP32 keeps state, gradients, limiter and fluxes in float, sums each cell's face
 * fluxes with a compensated (two-sum) accumulator, and keeps geometry precompute and the
 * residual-norm reduction in double. */
enum hcfd_precision { HCFD_FP64 = 0, HCFD_FP32 = 1 };

/* Cell renumbering applied by hcfd_mesh_renumber. */
enum hcfd_numbering {
    HCFD_NUMBER_NATURAL = 0, HCFD_NUMBER_RANDOM = 1, HCFD_NUMBER_RCM = 2, HCFD_NUMBER_MORTON = 3
};

/* ---- meshes ------------------------------------------------------------------------- */

/* The public raw arrays of the reference's Mesh (includes/Mesh.hpp:4-22).  Cells include
 * the boundary ghost cells (the mesh's line elements); faces are grouped by colour in
 * coloff order, interior colour(s) first, then NBCcol boundary colours, and every boundary
 * face has its ghost cell on the right (fc_con[2f+1]).  cc_off/cc_con may be NULL. */
typedef struct hcfd_mesh_view {
    int dim, Nn, Ncol, NBCcol, Nc, Nf;
    const int*    coltag;   /* [Ncol]            */
    const int*    coloff;   /* [Ncol+1]          */
    const double* nodes;    /* [Nn*dim]          */
    const int*    fn_con;   /* [2*Nf]            */
    const int*    fc_con;   /* [2*Nf]            */
    const int*    cn_off;   /* [Nc+1]            */
    const int*    cn_con;   /* [cn_off[Nc]]      */
    const int*    cc_off;   /* [Nc+1] or NULL    */
    const int*    cc_con;   /* [cc_off[Nc]]      */
} hcfd_mesh_view;

typedef struct hcfd_mesh hcfd_mesh;   /* host mesh owned by the library */

/* Replaces Mesh::Mesh(const char* fname) (src/Mesh.cpp:7-54).  Unlike the reference it
 * checks the file: a missing, truncated or inconsistent .hmsh gives HCFD_EIO/HCFD_EINVAL. */
int  hcfd_mesh_load(const char* path, hcfd_mesh** out);
/* Writes the .hmsh layout of interface/Mesh.py:441-463 (header, names, coltag, coloff,
 * nodes, fn_con, fc_con, cn_off, cn_con, cc_off, cc_con, c_ctypes). */
int  hcfd_mesh_write(const hcfd_mesh* m, const char* path);
/* Fills *v with pointers into m (valid until m is freed or renumbered): the arrays the
 * reference's Mesh exposes as public members (includes/Mesh.hpp:4-13). */
int  hcfd_mesh_view_of(const hcfd_mesh* m, hcfd_mesh_view* v);
/* The CSR cell->face table of Mesh::compute_cf_con (src/Mesh.cpp:88-117): the faces of
 * cell c, in increasing face index, are cf_con[cf_off[c] .. cf_off[c+1]). */
int  hcfd_mesh_cf(const hcfd_mesh* m, const int** cf_off, const int** cf_con);
/* Physical name k (the reference's Mesh::pnames, src/Mesh.cpp:70-86) or NULL. */
const char* hcfd_mesh_pname(const hcfd_mesh* m, int k);
/* Replaces Mesh::~Mesh (src/Mesh.cpp:54-68). */
void hcfd_mesh_free(hcfd_mesh* m);

/* Supersonic-wedge generator (the mesh family of the reference's wedge.hmsh, produced
 * here directly instead of through gmsh and interface/Mesh.py).  Domain x in [0, length],
 * top wall y = height, bottom wall y_b(x) = max(0, (x - x_ramp) tan(theta)).  nx x ny
 * nodes mapped vertically between y_b and the top; interior nodes jittered by
 * U(-jitter, jitter) times the local spacing in x and y; each quad split into two
 * triangles along a diagonal picked by a seeded coin flip; one ghost line cell per
 * boundary edge.  Colours: 0 interior, 1 "upper", 2 "lower", 3 "inlet", 4 "outlet"
 * (the colour tags of the reference's wedge.hmsh, driven by src/Test.cpp:64).  Cells are
 * then renumbered by `numbering` (the random permutation uses `seed` too). */
typedef struct hcfd_wedge_spec {
    int      nx, ny;
    double   length, height, x_ramp, theta_deg, jitter;
    uint64_t seed;
    int      numbering;   /* enum hcfd_numbering */
} hcfd_wedge_spec;
int  hcfd_mesh_generate_wedge(const hcfd_wedge_spec* spec, hcfd_mesh** out);
/* Renumbers the cells (ghosts included) and re-sorts faces inside each colour by
 * (min cell, max cell), with interior faces oriented CL < CR and boundary faces keeping
 * the ghost on the right: the face order interface/Mesh.py:321-378 produces. */
int  hcfd_mesh_renumber(hcfd_mesh* m, int numbering, uint64_t seed);

/* ---- solver ------------------------------------------------------------------------- */

typedef struct hcfd_params {
    double gma;         /* ratio of specific heats, Flux(nvars, gma, domain) (includes/Base/Flux.hpp:9) */
    int    limiter;     /* enum hcfd_limiter                                                 */
    double venkat_K;    /* Venkatakrishnan constant (limiter == HCFD_LIMITER_VENKAT)         */
    int    precision;   /* enum hcfd_precision                                               */
    int    block;       /* compute threads per block of the step kernels (multiple of 32; at
                           most 256 for the tiled kernels), 0 = 256 for the per-cell kernels
                           and one thread per tile cell for the tiled kernels               */
    int    kernel;      /* enum hcfd_kernel                                                  */
    int    tile;        /* cells per tile of the tiled kernels (32..512, multiple of 32); 0 = see tile2 */
    int    keep_numbering; /* 1: keep the input cell order on the device instead of the Morton order */
    long long freeze_limiter_after; /* limiter freezing (not in the reference): steps 1..N compute
                           the limiter, later steps reuse step N's limiter values with fresh
                           gradients, counted from hcfd_gpu_initialise; 0 = never        */
    int    tile2;       /* cells per tile of pass 2 (32..512, multiple of 32); 0 = `tile` when
                           that is given; with neither given, pass 1 / pass 2 tiles are
                           224 / 192 cells in FP64 and 256 / 128 in FP32 (smaller where a
                           tiling does not fit shared memory)                            */
} hcfd_params;

/* Step kernels.  HCFD_KERNEL_TILED (default): persistent CTAs stage tiles of cells, their
 * faces and their halo in shared memory (TMA bulk copies) and compute each face flux once
 * per tile.  HCFD_KERNEL_CELL: one thread per cell gathering its faces from global memory.
 * Both form every per-cell sum in the same order and give the same results. */
enum hcfd_kernel { HCFD_KERNEL_TILED = 0, HCFD_KERNEL_CELL = 1 };

typedef struct hcfd_step_stats {
    double dt;          /* dt of the last step (minimum local dt under HCFD_LOCAL_CFL)       */
    double res_l2;      /* L2 density residual of the last step, sqrt(sum R_rho^2 / Nreal)   */
    double res_first;   /* residual of the first step this handle took                       */
    long long steps;    /* steps taken by this handle since hcfd_gpu_initialise              */
    int    nonfinite;   /* 1 if the last step produced a NaN or Inf residual                 */
} hcfd_step_stats;

typedef struct hcfd_solver hcfd_solver;

/* Replaces Domain(Mesh&) + GaussGreen(const Domain&) + Limiter(const Domain&) +
 * Flux(nvars, gma, const Domain&) + Euler(nvars, Domain&, ...) (includes/Base/Domain.hpp:26,
 * GradientSchemes.hpp:8, Limiters.hpp:8, Flux.hpp:9, TimeIntegrators.hpp:13): uploads the
 * mesh, computes the geometry on the device in double (src/Base/Domain.cpp:4-154, with
 * zero_bc_iv as the Euler constructor applies it, src/Base/Euler.cpp:24) and allocates
 * the state. */
int  hcfd_gpu_create(const hcfd_mesh_view* mesh, const hcfd_params* params, hcfd_solver** out);
/* Replaces Euler::gather_BCs(const BCtype* BCmap, const double QBC[][NVARS])
 * (src/Base/Euler.cpp:42-60): boundary colour k takes type bcmap[coltag[colour]] and the
 * primitive state qbc[4*k .. 4*k+3]. */
int  hcfd_gpu_gather_bcs(hcfd_solver* s, const int* bcmap, int nbcmap, const double* qbc);
/* Replaces Euler::initialise(const double QIC[NVARS]) (src/Base/Euler.cpp:62-77). */
int  hcfd_gpu_initialise(hcfd_solver* s, const double* qic);
/* Runs nsteps iterations of the body of Euler::run's loop (src/Base/Euler.cpp:86-96):
 * gradient, limiter, ghost gradients/limiter, flux, U += dt R, ghost cells.  dt_or_cfl is
 * dt under HCFD_FIXED_DT and the CFL number otherwise.  Enqueued on the handle's stream;
 * when stats is non-NULL the call waits and fills it. */
int  hcfd_gpu_step(hcfd_solver* s, int nsteps, int time_mode, double dt_or_cfl, hcfd_step_stats* stats);
/* Euler::compute_prims + copy-out (src/Base/Euler.cpp:115-136): prims != 0 gives
 * (rho, u, v, p), else the conservative state.  out[v] holds Nc doubles. */
int  hcfd_gpu_download(hcfd_solver* s, int prims, double* const* out);
/* Overwrites the conservative state from 4 host arrays of Nc doubles (checkpoint
 * restore; no reference counterpart). */
int  hcfd_gpu_upload(hcfd_solver* s, const double* const* in);
/* Checkpoint and resume (no reference counterpart: the reference's only output is the .hsln
 * snapshot of primitive variables, src/Euler.cpp:99-103, whose round trip to conservative
 * variables is inexact, and it has no reader).  hcfd_gpu_checkpoint writes the conservative
 * state of every cell (input numbering, doubles; FP32 values widen exactly), the step
 * statistics and, with limiter freezing, the recorded limiter values.  hcfd_gpu_restore loads
 * such a file into a solver made for the same mesh with the same parameters (BCs gathered):
 * the following steps are bit-identical to the uninterrupted solve.  HCFD_EIO for a file
 * that is not a checkpoint, HCFD_EINVAL for one of another mesh size, precision or freezing
 * setting.  hcfd_checkpoint_info reads a checkpoint's header (no GPU needed). */
/* Output without stopping the steps (no reference counterpart: Writer::write_soln,
 * src/Writer.cpp:22-39, runs between steps while the loop waits).  hcfd_gpu_snapshot converts
 * the current state (prims != 0: primitive) into a device staging buffer on the handle's
 * stream and copies it into the 4 host arrays of Nc doubles on a second stream, then returns
 * a ticket at once: later steps run while the copy is in flight.  Page-locked host arrays
 * (hcfd_host_pin) are needed for the copy to overlap; with pageable ones the call returns
 * only when the copy has landed.  hcfd_snapshot_wait blocks until the host arrays hold the
 * snapshot; it touches only the ticket, so a writer thread may call it while another thread
 * steps the solver.  hcfd_snapshot_free waits, then releases the ticket.  The first snapshot
 * allocates the staging buffer, a stream and an event. */
typedef struct hcfd_snapshot hcfd_snapshot;
int  hcfd_gpu_snapshot(hcfd_solver* s, int prims, double* const* host, hcfd_snapshot** ticket);
int  hcfd_snapshot_wait(hcfd_snapshot* t);
void hcfd_snapshot_free(hcfd_snapshot* t);
int  hcfd_gpu_checkpoint(hcfd_solver* s, const char* path);
int  hcfd_gpu_restore(hcfd_solver* s, const char* path);
int  hcfd_checkpoint_info(const char* path, int* Nc, int* precision, long long* steps, int* has_limiter);
/* Waits for the handle's stream; returns HCFD_ENONFINITE if a step produced a NaN/Inf (no
 * reference counterpart: the reference steps synchronously and never checks for NaN). */
int  hcfd_gpu_sync(hcfd_solver* s);
/* Statistics of the steps taken so far (waits for the stream; no reference counterpart:
 * the reference computes no residual). */
int  hcfd_gpu_stats(hcfd_solver* s, hcfd_step_stats* stats);
/* Failure injection for tests of the bounded waits (no reference counterpart: the reference
 * has no device and no waits).  Every wait of the tiled step kernels gives up after `polls`
 * polls (0 restores the default, 2^22; at most 2^30); with skip_tile >= 0 the staging warp
 * arms and copies nothing for that tile, so the wait for it runs out with no copy in flight.
 * The next step then returns HCFD_ETIMEOUT with the state partly stepped; the kernels leave
 * no copy in flight and the context stays usable: hcfd_gpu_initialise clears the error, and
 * with the hook reset (polls 0, skip_tile -1) the handle steps normally again. */
int  hcfd_gpu_test_waits(hcfd_solver* s, unsigned polls, int skip_tile);
/* Wall pressure coefficient (p_CL - p_inf) / (0.5 rho_inf |u_inf|^2) on the faces of one
 * colour, in face order; *n gets the face count.  No reference counterpart. */
int  hcfd_gpu_wall_cp(hcfd_solver* s, int colour, double rho_inf, double p_inf, double speed_inf,
                      double* out, int* n);
/* Mesh facts as the solver sees them: Nc, Nf, number of real (non-ghost) cells, the
 * face slots per cell of the step kernels (no reference counterpart). */
int  hcfd_gpu_info(hcfd_solver* s, int* Nc, int* Nf, int* Nreal, int* slots);
/* Per-kernel timing with CUDA events on the handle's stream (the reference times only whole
 * runs, with clock(), src/Test.cpp:72-74).  enable = N > 0 starts
 * recording the two step kernels' launches of every N-th step (N > 1 keeps the events'
 * own cost out of most steps); 0 stops.  hcfd_gpu_profile_read returns the summed
 * milliseconds and launch counts of the recorded launches since enabling. */
int  hcfd_gpu_profile(hcfd_solver* s, int enable);
int  hcfd_gpu_profile_read(hcfd_solver* s, double* ms_pass1, long long* n_pass1,
                           double* ms_pass2, long long* n_pass2);
/* Runs nsteps steps as hcfd_gpu_step does and waits; *ms gets the device time between two
 * CUDA events recorded on the handle's stream before the first and after the last launch.
 * No reference counterpart (the reference times whole runs with clock(), src/Test.cpp:72-74). */
int  hcfd_gpu_step_timed(hcfd_solver* s, int nsteps, int time_mode, double dt_or_cfl, double* ms);
/* Number of kernel launches one step issues (the two passes; no reference counterpart). */
int  hcfd_gpu_launches_per_step(hcfd_solver* s);
/* Replaces the Euler destructor (src/Base/Euler.cpp:27-40) and those of the objects
 * hcfd_gpu_create stands in for: frees the handle's device memory, stream and graphs. */
void hcfd_gpu_destroy(hcfd_solver* s);

/* Page-locks a caller-owned host range (cudaHostRegister) so that hcfd_gpu_upload and
 * hcfd_gpu_download from and to it run as direct DMA; hcfd_host_unpin releases it (no
 * reference counterpart). */
int  hcfd_host_pin(void* p, size_t bytes);
int  hcfd_host_unpin(void* p);

/* Builds the tiled kernels' execution plan for a mesh on the host (no device needed) and
 * checks every index the kernels derive from it: local cell indices inside the staged
 * range, each flux slot written by exactly one face entry, slots in increasing face order,
 * bulk-copy sizes and offsets multiples of 16 bytes.  info (8 values, may be NULL): tiles,
 * max halo, max face entries, entries, faces computed once (both cells in one tile), cut
 * face entries, slots per cell, total halo cells.  No reference counterpart. */
int  hcfd_plan_check(const hcfd_mesh_view* mesh, int tile, int keep_numbering, long long* info);

/* ---- batched and served solves: many meshes in one device arena --------------------- */

/* No counterpart in the reference (it solves one mesh per process).  An arena packs many
 * meshes (instances) into one flat set of device arrays sized from an HBM budget; each
 * admitted mesh gets contiguous ranges (per-instance offsets), its own BC table, dt or CFL
 * number and statistics, and all active instances advance together through the tiled step
 * kernels, a chunk of steps replayed as one CUDA graph.  An instance's arithmetic does not
 * depend on what else is in the arena: its state is the same alone and in the mix. */
typedef struct hcfd_arena hcfd_arena;
typedef struct hcfd_arena_params {
    size_t hbm_budget;      /* bytes of device memory the arena's arrays may use            */
    int    precision;       /* enum hcfd_precision                                          */
    int    limiter;         /* enum hcfd_limiter                                            */
    double venkat_K;
    double gma;
    int    time_mode;       /* enum hcfd_time_mode, shared by all instances                 */
    int    tile;            /* cells per tile (32..256, multiple of 32), 0 = 128            */
    int    slots;           /* faces per cell: 3 (triangles) or 4 (quads), 0 = 3            */
    int    max_instances;   /* instance slots                                               */
    long long freeze_limiter_after; /* as in hcfd_params, counted per instance from admission */
} hcfd_arena_params;
typedef struct hcfd_arena_info_t {
    size_t cell_capacity, cells_used, face_capacity, faces_used;
    int active, active_tiles;
    long long steps;
    int tile;
} hcfd_arena_info_t;

int  hcfd_arena_create(const hcfd_arena_params* params, hcfd_arena** out);
/* Admits one mesh with its BC map and states (as hcfd_gpu_gather_bcs), its initial state
 * (as hcfd_gpu_initialise) and its dt (fixed mode) or CFL number.  Returns HCFD_EAGAIN when
 * the budget, a free range or an instance slot is missing: retry after a release. */
int  hcfd_arena_admit(hcfd_arena* a, const hcfd_mesh_view* mesh, const int* bcmap, int nbcmap, const double* qbc,
                      const double* qic, double dt_or_cfl, int* slot);
/* The same admission in two halves, so that a server can build tile plans on worker
 * threads while another thread steps the arena.  hcfd_arena_prepare does the host work
 * (cell->face table, Morton order, tile plan, BC table); it reads only the arena's fixed
 * parameters, so any number of threads may call it at once.  The mesh arrays must stay
 * valid until the admission is freed.  hcfd_arena_admit_prepared claims the ranges and
 * enqueues the uploads and the set-up kernels on the arena's admission stream, behind which
 * the steps already enqueued keep running; the instance joins the active set at the next
 * hcfd_arena_step (poll, fetch, checkpoint, restore and release wait for pending admissions
 * on the device).  On HCFD_EAGAIN the admission stays valid for a later try. */
typedef struct hcfd_admission hcfd_admission;
int  hcfd_arena_prepare(const hcfd_arena* a, const hcfd_mesh_view* mesh, const int* bcmap, int nbcmap,
                        const double* qbc, const double* qic, double dt_or_cfl, hcfd_admission** out);
int  hcfd_arena_admit_prepared(hcfd_arena* a, const hcfd_admission* adm, int* slot);
/* Arena cells (whole tiles) the admission will take. */
size_t hcfd_admission_cells(const hcfd_admission* adm);
void hcfd_admission_free(hcfd_admission* adm);
/* Advances every active instance by nsteps steps (enqueued; returns without waiting). */
int  hcfd_arena_step(hcfd_arena* a, int nsteps);
/* Waits, then reports up to max active instances: their slots and step statistics. */
int  hcfd_arena_poll(hcfd_arena* a, int max, int* slots, hcfd_step_stats* stats, int* n);
/* Copies one instance's state (prims != 0: primitive) to 4 host arrays of its Nc doubles. */
int  hcfd_arena_fetch(hcfd_arena* a, int slot, int prims, double* const* out);
/* An instance's exact snapshot (hcfd_gpu_checkpoint's format), and its restore into an
 * admitted instance of the same mesh, for preempting a served solve and resuming it later
 * (here or in another arena) with the same results. */
int  hcfd_arena_checkpoint(hcfd_arena* a, int slot, const char* path);
int  hcfd_arena_restore(hcfd_arena* a, int slot, const char* path);
/* Retires an instance and frees its ranges for later admissions. */
int  hcfd_arena_release(hcfd_arena* a, int slot);
int  hcfd_arena_info(hcfd_arena* a, hcfd_arena_info_t* info);
void hcfd_arena_destroy(hcfd_arena* a);

/* ---- one step without device allocation -------------------------------------------- */

/* No counterpart in the reference.  For callers that cannot call cudaMalloc: a framework
 * that owns all device memory through its own pool, a caller that must not let a library
 * allocate (cudaMalloc and cudaFree can synchronise the device), or a loop with a fixed
 * memory budget.  The caller owns every input and output in its own device buffers; the
 * only other memory the step needs (the limited gradients between its two passes and the
 * reduction slots) is a static device array of the library, sized for at most
 * HCFD_NOALLOC_MAX_CELLS cells (about 4 MiB, held on every GPU that loads the library until
 * the process exits).  Larger meshes are rejected with HCFD_EINVAL. */
#define HCFD_NOALLOC_MAX_CELLS 65536

typedef struct hcfd_noalloc_mesh {
    int Nc;                 /* cells, ghosts included (1..HCFD_NOALLOC_MAX_CELLS)                 */
    int Nf;                 /* faces                                                              */
    int F_BC;               /* first boundary face (faces F_BC..Nf-1 have a ghost on the right)   */
    int slots;              /* face slots per cell: 3, 4 or 8                                     */
    const int* slot;        /* device, slots x Nc int pairs, slot-major: slot k of cell c at
                               2 (k Nc + c): {face f if c is the face's left cell, else ~f;
                               the other cell}; unused slots {-1, -1}; a ghost cell's first slot
                               is unused.  Each cell's faces in increasing face index.          */
    const double* geo;      /* device, Nf x 8: nx, ny, length, If, rLx, rLy, rRx, rRy (the
                               layout of the reference's Domain face arrays,
                               includes/Base/Domain.hpp:15-24)                                    */
    const double* iv;       /* device, Nc: 1/area, 0 for ghost cells                               */
    int nbc;                /* boundary colours (0..16)                                           */
    const int* bc_first;    /* host, nbc + 1: first face of each boundary colour, then Nf;
                               non-decreasing, bc_first[0] = F_BC, bc_first[nbc] = Nf
                               (nbc = 0 requires F_BC = Nf)                                       */
    const int* bc_type;     /* host, nbc: enum hcfd_bctype                                        */
    const double* bc_state; /* host, nbc x 4: primitive (rho, u, v, p)                            */
    double gma;
    int limiter;            /* enum hcfd_limiter                                                  */
    double venkat_K;
} hcfd_noalloc_mesh;

/* New entry point, no reference counterpart.  One step (HCFD_FIXED_DT or HCFD_GLOBAL_CFL)
 * from U_in to U_out, both caller-owned device buffers of 4 Nc doubles whose address ranges
 * must not overlap (HCFD_EINVAL otherwise), laid out as two planes of pairs: plane 0 holds
 * (rho, rho u) of cells 0..Nc-1, plane 1 (at offset 2 Nc) holds (rho v, E).  Work is
 * enqueued on `stream` (a cudaStream_t, NULL for the default stream).  When dt_used or
 * res_l2 is non-NULL the call waits for the stream, reports the step's dt and L2 density
 * residual, and returns HCFD_ENONFINITE if the step produced a NaN or Inf; with both NULL
 * it returns without waiting and nothing checks the new state for NaN or Inf.  Allocates
 * nothing: no cudaMalloc, cudaFree or allocating library call.
 * The first call on each device (and again the first call after the device's context was
 * replaced, e.g. by cudaDeviceReset) looks up the device address of the static scratch;
 * make that first call before any stream capture.  All calls share the one scratch array,
 * which keeps the last call's contents: calls that overlap on the GPU (other streams, other
 * threads) race and must be serialised by the caller. */
int  hcfd_step_noalloc(const hcfd_noalloc_mesh* mesh, const double* U_in, double* U_out, int time_mode,
                       double dt_or_cfl, void* stream, double* dt_used, double* res_l2);

/* ---- output ------------------------------------------------------------------------- */

/* Replaces Writer::write_soln (src/Writer.cpp:22-39): writes int32 Nc, nvars, nchars,
 * the NUL-terminated names, then nvars x Nc doubles to `path` (the caller forms the
 * reference's "<fname>_<runcount>.hsln" name). */
int  hcfd_write_hsln(const char* path, int nvars, const char* const* varnames, int Nc,
                     const double* const* arrs);

/* ---- devices ------------------------------------------------------------------------ */

/* Makes `device` the calling thread's current CUDA device for the handles it creates
 * afterwards (one process per GPU; a handle stays on the device it was created on).
 * *count, if non-NULL, gets the number of visible devices.  No reference counterpart (the
 * reference is a single-threaded CPU program), nor for hcfd_device_sync. */
int  hcfd_set_device(int device, int* count);
/* Waits for all work on the current device (cudaDeviceSynchronize). */
int  hcfd_device_sync(void);
/* Free and total device memory of the current device in bytes (cudaMemGetInfo), for sizing
 * an arena's HBM budget.  No reference counterpart. */
int  hcfd_device_mem_info(size_t* free_bytes, size_t* total_bytes);

/* ---- errors ------------------------------------------------------------------------- */
/* Text of the calling thread's last failure.  No reference counterpart: the reference
 * reports no errors (no return codes or exceptions; fopen and fread results unchecked,
 * src/Mesh.cpp:9-45, src/Writer.cpp:25). */
const char* hcfd_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* HCFD_GPU_H */
