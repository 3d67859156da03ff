// Internal declarations shared by the host and device translation units of libhcfd_gpu.
#pragma once
#include "hcfd_gpu.h"

#include <string>
#include <vector>

namespace hcfd {

// Thread-local text behind hcfd_last_error(); every failing entry point sets it.
int fail(int code, const std::string& msg);
void clear_error();

}  // namespace hcfd

// Host mesh: the public arrays of the reference's Mesh (includes/Mesh.hpp:4-22) plus the
// cell->face table it derives (src/Mesh.cpp:88-117) and the c_ctypes the Python importer
// writes (interface/Mesh.py:463).
struct hcfd_mesh {
    int dim = 2, Nn = 0, Ncol = 0, NBCcol = 0, Nc = 0, Nf = 0;
    std::vector<std::string> pnames;
    std::vector<int> coltag, coloff;
    std::vector<double> nodes;
    std::vector<int> fn_con, fc_con, cn_off, cn_con, cc_off, cc_con, c_ctypes;
    std::vector<int> cf_off, cf_con;
};

namespace hcfd {
// Checks index ranges and the colour/ghost conventions of a mesh view.  Returns HCFD_OK or
// HCFD_EINVAL with the reason recorded.
int validate_view(const hcfd_mesh_view& v);
// Builds cf_off/cf_con exactly as Mesh::compute_cf_con does (faces of each cell in
// increasing face index).
void build_cf(int Nc, int Nf, const int* fc_con, std::vector<int>& cf_off, std::vector<int>& cf_con);

// Execution plan of the tiled step kernels (hcfd_plan.cpp).
struct TilePlan {
    int B = 256, W = 3, Wp = 4, ntiles = 0, Hmax = 0, Fmax = 0;
    std::vector<int> foff, hoff, halo, efid;
    std::vector<short> meta, cslot;
};
// Internal cell order: cells sorted by the Morton key of their vertex-average centre.
// Returns perm with perm[internal] = input index.
std::vector<int> morton_order(const hcfd_mesh_view& v);
// face_groups: number each tile's face entries so that every run of 8 consecutive entries
// reads cells in distinct shared-memory bank groups on each side where it can (the entry
// order pass 2's face phase reads in); pass 1, which reads entries through its cells' slots,
// keeps the order in which its cells meet their faces.
int build_tile_plan(const hcfd_mesh_view& v, const std::vector<int>& cf_off, const std::vector<int>& cf_con,
                    const std::vector<char>& ghost, const std::vector<int>& perm, int F_BC,
                    const std::vector<int>& bc_first, int B, int W, TilePlan& P, bool face_groups = false);
}  // namespace hcfd

namespace hcfd {
// Checkpoint file of one solve (hcfd_gpu_checkpoint / hcfd_arena_checkpoint): this header,
// then the conservative state of every cell, variable-major, in the input numbering, as
// doubles (FP32 values widen exactly), then, with limiter freezing, the recorded limiter
// values in the same layout.
struct CkptHeader {
    char magic[8];               // "HCFDCKP1"
    int version;                 // 1
    int precision;               // enum hcfd_precision of the solve
    int Nc;
    int has_phiF;
    long long steps;
    double res2_first, res2_last, dt_last;
    int nonfinite, pad;
};
int ckpt_write(const char* path, const CkptHeader& h, const std::vector<double>& U, const std::vector<double>* phiF);
int ckpt_read(const char* path, CkptHeader& h, std::vector<double>* U, std::vector<double>* phiF);
}  // namespace hcfd

