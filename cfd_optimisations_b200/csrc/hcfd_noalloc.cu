// hcfd_step_noalloc: one time step of the per-cell step kernels for callers that cannot
// allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not allowed or not wanted — a host
// framework that owns every byte of device memory through its own pool, a caller building
// a stream that must not synchronise the device (cudaMalloc/cudaFree can), or a real-time
// loop with a fixed memory budget.  Such a caller owns the inputs and outputs (state, face
// records, cell->face slots, inverse areas) in its own device buffers; this entry point
// adds no allocation of any kind.  The one buffer the step needs besides them — the limited
// gradients that pass 1 writes and pass 2 reads, plus the reduction slots — is the static
// device array below, sized for at most HCFD_NOALLOC_MAX_CELLS cells.  Every GPU that loads
// the library holds that array (about 4 MiB) until the process exits.
#include "hcfd_internal.hpp"
#include "hcfd_kernels.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

using hcfd::fail;

namespace {

constexpr int kBlock = 256;
constexpr int kMaxBlocks = (HCFD_NOALLOC_MAX_CELLS + kBlock - 1) / kBlock;

// Byte layout of the scratch array (offsets are multiples of 256).
constexpr size_t kPhiG = 0;                                                   // Grad8<double> planes
constexpr size_t kPartial = kPhiG + (size_t) 64 * HCFD_NOALLOC_MAX_CELLS;     // double[kMaxBlocks]
constexpr size_t kDtmin = kPartial + ((sizeof(double) * kMaxBlocks + 255) & ~(size_t) 255);  // u64[2]
constexpr size_t kCounter = kDtmin + 256;                                     // unsigned int
constexpr size_t kErr = kCounter + 128;                                       // unsigned int (checked build)
constexpr size_t kStats = kCounter + 256;                                     // StepStats
constexpr size_t kScratchBytes = kStats + 256;

// The scratch.  In host code `g_noalloc_scratch` names a host-side stand-in, not device
// memory: kernels get the device address taken by cudaGetSymbolAddress at set-up.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// The device address of the scratch belongs to a CUDA context: after cudaDeviceReset (or
// any other end of the context) the device holds a new copy at a new address.  The address
// is therefore cached per device together with the unique id of the context it was taken in
// (cuCtxGetId, ids are never reused within a process) and looked up again when the current
// context's id differs.  The two driver calls come through cudaGetDriverEntryPointByVersion,
// so the library needs no link against libcuda.
constexpr int kMaxDevices = 64;
struct ScratchAddr {
    unsigned long long ctx_id;   // 0: not looked up yet
    unsigned char* addr;
};
ScratchAddr g_addr[kMaxDevices] = {};
std::mutex g_addr_mu;
PFN_cuCtxGetCurrent_v4000 g_ctx_current = nullptr;
PFN_cuCtxGetId_v12000 g_ctx_id = nullptr;
bool g_entry_points_tried = false;

// Id of the calling thread's current context, 0 when there is none or it cannot be told.
unsigned long long current_ctx_id() {
    if (!g_entry_points_tried) {
        g_entry_points_tried = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f);
    }
    if (!g_ctx_current || !g_ctx_id) return 0;
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (g_ctx_current(&c) != CUDA_SUCCESS || !c || g_ctx_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Clears what must start at zero (and the dt minimum at +inf) on every call.
__global__ void noalloc_reset_kernel(unsigned long long* dtmin, unsigned int* counter, unsigned int* err,
                                     hcfd::StepStats* stats) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        dtmin[0] = 0x7FF0000000000000ULL;
        dtmin[1] = 0x7FF0000000000000ULL;
        *counter = 0u;
        *err = 0u;
        hcfd::StepStats z{};
        *stats = z;
    }
}

template <int W>
void launch(const hcfd::StepArgs<double>& a, cudaStream_t st) {
    const int grid = (a.Nc + kBlock - 1) / kBlock;
    hcfd::pass1_kernel<double, W><<<grid, kBlock, 0, st>>>(a);
    hcfd::pass2_kernel<double, W, false><<<grid, kBlock, 0, st>>>(a);
}

}  // namespace

extern "C" int hcfd_step_noalloc(const hcfd_noalloc_mesh* m, const double* U_in, double* U_out, int time_mode,
                                 double dt_or_cfl, void* stream, double* dt_used, double* res_l2) {
    hcfd::clear_error();
    if (!m || !U_in || !U_out || !m->slot || !m->geo || !m->iv)
        return fail(HCFD_EINVAL, "step_noalloc: null argument");
    if (m->Nc <= 0 || m->Nc > HCFD_NOALLOC_MAX_CELLS)
        return fail(HCFD_EINVAL, "step_noalloc: Nc must be in 1.." + std::to_string(HCFD_NOALLOC_MAX_CELLS) +
                                     " (the size of the static scratch)");
    {
        // pass 2 writes U_out while other cells still read U_in: the ranges must be disjoint
        const uintptr_t a0 = reinterpret_cast<uintptr_t>(U_in), b0 = reinterpret_cast<uintptr_t>(U_out);
        const uintptr_t n = sizeof(double) * 4 * (uintptr_t) m->Nc;
        if (a0 < b0 + n && b0 < a0 + n) return fail(HCFD_EINVAL, "step_noalloc: U_in and U_out overlap");
    }
    if (m->Nf <= 0 || m->F_BC < 0 || m->F_BC > m->Nf || (m->slots != 3 && m->slots != 4 && m->slots != 8) ||
        m->nbc < 0 || m->nbc > hcfd::MAXBC || (m->nbc > 0 && (!m->bc_first || !m->bc_type || !m->bc_state)) ||
        !(m->gma > 1.0) || (m->limiter != HCFD_LIMITER_BJ && m->limiter != HCFD_LIMITER_VENKAT) ||
        time_mode < HCFD_FIXED_DT || time_mode > HCFD_GLOBAL_CFL || !std::isfinite(dt_or_cfl) || dt_or_cfl < 0)
        return fail(HCFD_EINVAL, "step_noalloc: bad argument");
    // The boundary table must cover exactly the boundary faces F_BC..Nf-1, in order: a face
    // outside it would be refreshed with another colour's type and state.
    if (m->nbc == 0 ? m->F_BC != m->Nf : (m->bc_first[0] != m->F_BC || m->bc_first[m->nbc] != m->Nf))
        return fail(HCFD_EINVAL, "step_noalloc: the boundary colours must cover faces F_BC..Nf-1");
    for (int b = 0; b < m->nbc; b++)
        if (m->bc_first[b + 1] < m->bc_first[b])
            return fail(HCFD_EINVAL, "step_noalloc: bc_first must not decrease");

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(HCFD_ECUDA, std::string("step_noalloc: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(HCFD_EINVAL, "step_noalloc: device index too large");
    unsigned char* base;
    {
        // Once per device and context, with that device current: the device address of the
        // scratch.  Where the context id cannot be read, the address is looked up on every
        // call (a host-side lookup; it allocates nothing).
        std::lock_guard<std::mutex> lk(g_addr_mu);
        const unsigned long long id = current_ctx_id();
        if (id == 0 || g_addr[dev].ctx_id != id) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return fail(HCFD_ECUDA, std::string("step_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            // the lookup makes the device's context current if none was: take its id now
            g_addr[dev].ctx_id = current_ctx_id();
            g_addr[dev].addr = static_cast<unsigned char*>(p);
        }
        base = g_addr[dev].addr;
    }

    hcfd::BCTable bc{};
    bc.nbc = m->nbc;
    for (int b = 0; b < m->nbc; b++) {
        bc.F1[b] = m->bc_first[b];
        bc.type[b] = m->bc_type[b];
        if (bc.type[b] < HCFD_SYMMETRY || bc.type[b] > HCFD_SUBOUTLET) return fail(HCFD_EINVAL, "step_noalloc: bad BC type");
        const double* q = m->bc_state + 4 * b;
        for (int v = 0; v < 4; v++) bc.QBC[b][v] = q[v];
        // primitive -> conservative, BoundaryCondition::init (src/Base/BoundaryConditions/Base.cpp:18-22)
        bc.UBC[b][0] = q[0];
        for (int v = 1; v < 4; v++) bc.UBC[b][v] = q[0] * q[v];
        bc.UBC[b][3] = q[3] / (m->gma - 1) + 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2]);
    }
    bc.F1[m->nbc] = m->nbc > 0 ? m->bc_first[m->nbc] : m->Nf;

    hcfd::StepArgs<double> a;
    a.U = reinterpret_cast<const hcfd::Cell4<double>*>(U_in);
    a.Unew = reinterpret_cast<hcfd::Cell4<double>*>(U_out);
    a.phiG = reinterpret_cast<hcfd::Grad8<double>*>(base + kPhiG);
    a.geo = reinterpret_cast<const hcfd::FaceGeo<double>*>(m->geo);
    a.slot = reinterpret_cast<const int2*>(m->slot);
    a.iv = m->iv;
    a.dtmin = reinterpret_cast<unsigned long long*>(base + kDtmin);
    a.dtmin_next = a.dtmin + 1;
    a.partial = reinterpret_cast<double*>(base + kPartial);
    a.counter = reinterpret_cast<unsigned int*>(base + kCounter);
    a.stats = reinterpret_cast<hcfd::StepStats*>(base + kStats);
    a.Nc = m->Nc;
    a.F_BC = m->F_BC;
    a.limiter = m->limiter;
    a.time_mode = time_mode;
    a.gma = m->gma;
    a.venkat_K = m->venkat_K;
    a.dt_or_cfl = dt_or_cfl;
    a.bc = bc;
    a.phiF = nullptr;        // no limiter freezing here
    a.freeze_after = 0;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned int* d_err = reinterpret_cast<unsigned int*>(base + kErr);
    noalloc_reset_kernel<<<1, 32, 0, st>>>(a.dtmin, a.counter, d_err, a.stats);
    if constexpr (hcfd::kChecked) {
        // checked build: the caller's slot table is checked on the device before the step,
        // which is not launched when an id is out of range
        const long long n = (long long) m->slots * m->Nc;
        hcfd::check_slots_kernel<<<(int) std::min<long long>((n + 255) / 256, 1184), 256, 0, st>>>(
            a.slot, m->slots, m->Nc, m->Nf, d_err);
        unsigned int err = 0;
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&err, d_err, sizeof(err), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(HCFD_ECUDA, std::string("step_noalloc: ") + cudaGetErrorString(e));
        if (err & 4u) return fail(HCFD_EINVAL, "step_noalloc, checked build: a face or neighbour id was out of range");
    }
    switch (m->slots) {
    case 3: launch<3>(a, st); break;
    case 4: launch<4>(a, st); break;
    default: launch<8>(a, st); break;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(HCFD_ECUDA, std::string("step_noalloc: launch: ") + cudaGetErrorString(e));
    if (dt_used || res_l2) {
        hcfd::StepStats h{};
        e = cudaMemcpyAsync(&h, a.stats, sizeof(h), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(HCFD_ECUDA, std::string("step_noalloc: ") + cudaGetErrorString(e));
        const int nreal = m->Nc - (m->Nf - m->F_BC);
        if (dt_used) *dt_used = h.dt_last;
        if (res_l2) *res_l2 = nreal > 0 ? std::sqrt(h.res2_last / nreal) : 0.0;
        if (h.nonfinite) return fail(HCFD_ENONFINITE, "step_noalloc: a NaN or Inf appeared");
    }
    return HCFD_OK;
}
