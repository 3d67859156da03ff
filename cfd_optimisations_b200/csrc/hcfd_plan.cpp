// Host-side execution plan of the tiled step kernels.
//
// The device keeps cells in an internal order (a Morton curve over the cell centres by
// default, so that consecutive cells are close in space whatever the input numbering) and
// cuts that order into tiles of B consecutive cells.  For each tile the plan lists
//   - its halo: cells outside the tile that neighbour one of its real cells;
//   - its face entries: every face with a real tile cell on either side, once per tile,
//     with the local indices (tile cells 0..B-1, halo cells B..) of both cells, the flux
//     slots the entry feeds (local cell * W + position of the face in that cell's face
//     list), and the boundary-condition index of boundary faces;
//   - per tile cell and face position: the local entry index and the side of the cell.
// A cell's face positions follow its faces in increasing face index (the order of the
// reference's cell->face table, src/Mesh.cpp:88-117), so per-cell sums formed slot by
// slot add in the reference's order.
#include "hcfd_internal.hpp"

#include <algorithm>
#include <cstring>
#include <numeric>

namespace hcfd {

namespace {
unsigned long long spread16(unsigned long long x) {
    x &= 0xFFFFULL;
    x = (x | (x << 8)) & 0x00FF00FFULL;
    x = (x | (x << 4)) & 0x0F0F0F0FULL;
    x = (x | (x << 2)) & 0x33333333ULL;
    x = (x | (x << 1)) & 0x55555555ULL;
    return x;
}
}  // namespace

// Renumbers the real (non-padding) entries [e0, e0 + n) of tile t for pass 2's face phase,
// in which the 8 lanes of a quarter warp read the 16-byte cell and gradient chunks of 8
// consecutive entries' left cells, then of their right cells.  Those reads conflict in shared
// memory when two lanes read different cells of the same bank group (local cell index mod 8,
// every plane being a multiple of 128 bytes apart).  Entries are taken greedily into groups of
// 8: each pick comes from the non-empty (left mod 8, right mod 8) class that adds the fewest
// conflicts to the group (a cell already read in the group adds none), the fullest class first
// among equals.  Only the numbering changes: each cell's slots still list its faces in
// increasing face order, so every per-cell sum keeps its order.
static void group_entries(TilePlan& P, int t, int e0, int n, int nb) {
    if (n <= 8) return;
    std::vector<int> bucket_head[64];
    for (int e = 0; e < n; e++) {
        const short* m = &P.meta[4 * (size_t) (e0 + e)];
        bucket_head[(m[0] & 7) * 8 + (m[1] & 7)].push_back(e);
    }
    int pos[64] = {0};
    std::vector<int> order;
    order.reserve(n);
    while ((int) order.size() < n) {
        int ua[8], ub[8];
        for (int k = 0; k < 8; k++) ua[k] = ub[k] = -1;
        const int g = std::min(8, n - (int) order.size());
        for (int i = 0; i < g; i++) {
            int best = -1, bcost = 3, bleft = 0;
            for (int k = 0; k < 64; k++) {
                const int left = (int) bucket_head[k].size() - pos[k];
                if (left <= 0) continue;
                const short* m = &P.meta[4 * (size_t) (e0 + bucket_head[k][pos[k]])];
                const int a = m[0], b = m[1];
                const int cost = (ua[a & 7] >= 0 && ua[a & 7] != a) + (ub[b & 7] >= 0 && ub[b & 7] != b);
                if (cost < bcost || (cost == bcost && left > bleft)) { best = k; bcost = cost; bleft = left; }
            }
            const int e = bucket_head[best][pos[best]++];
            const short* m = &P.meta[4 * (size_t) (e0 + e)];
            if (ua[m[0] & 7] < 0) ua[m[0] & 7] = m[0];
            if (ub[m[1] & 7] < 0) ub[m[1] & 7] = m[1];
            order.push_back(e);
        }
    }
    std::vector<int> newpos(n);
    std::vector<int> efid(n);
    std::vector<short> meta(4 * (size_t) n);
    for (int i = 0; i < n; i++) {
        const int e = order[i];
        newpos[e] = i;
        efid[i] = P.efid[e0 + e];
        for (int k = 0; k < 4; k++) meta[4 * (size_t) i + k] = P.meta[4 * (size_t) (e0 + e) + k];
    }
    std::copy(efid.begin(), efid.end(), P.efid.begin() + e0);
    std::copy(meta.begin(), meta.end(), P.meta.begin() + 4 * (size_t) e0);
    short* cs = &P.cslot[(size_t) t * P.B * P.Wp];
    for (int c = 0; c < nb; c++)
        for (int k = 0; k < P.Wp; k++) {
            short& x = cs[(size_t) c * P.Wp + k];
            if (x >= 0) x = (short) ((newpos[x >> 1] << 1) | (x & 1));
        }
}

std::vector<int> morton_order(const hcfd_mesh_view& v) {
    double lo[2] = {1e300, 1e300}, hi[2] = {-1e300, -1e300};
    for (int i = 0; i < v.Nn; i++)
        for (int d = 0; d < 2; d++) { lo[d] = std::min(lo[d], v.nodes[2 * i + d]); hi[d] = std::max(hi[d], v.nodes[2 * i + d]); }
    std::vector<unsigned int> key(v.Nc);
    for (int c = 0; c < v.Nc; c++) {
        double x[2] = {0, 0};
        const int b = v.cn_off[c], e = v.cn_off[c + 1];
        for (int k = b; k < e; k++)
            for (int d = 0; d < 2; d++) x[d] += v.nodes[2 * v.cn_con[k] + d];
        unsigned long long q[2];
        for (int d = 0; d < 2; d++) {
            double t = (hi[d] > lo[d]) ? (x[d] / (e - b) - lo[d]) / (hi[d] - lo[d]) : 0.0;
            t = std::min(std::max(t, 0.0), 1.0);
            q[d] = (unsigned long long) (t * 65535.0);
        }
        key[c] = (unsigned int) (spread16(q[0]) | (spread16(q[1]) << 1));
    }
    std::vector<int> perm(v.Nc);
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return key[a] < key[b]; });
    return perm;
}

int build_tile_plan(const hcfd_mesh_view& v, const std::vector<int>& cf_off, const std::vector<int>& cf_con,
                    const std::vector<char>& ghost, const std::vector<int>& perm, int F_BC,
                    const std::vector<int>& bc_first, int B, int W, TilePlan& P, bool face_groups) {
    const int Nc = v.Nc;
    P.B = B;
    P.W = W;
    P.Wp = W;
    P.ntiles = (Nc + B - 1) / B;
    std::vector<int> iperm(Nc);
    for (int i = 0; i < Nc; i++) iperm[perm[i]] = i;
    auto bc_of = [&](int f) {
        int k = 0;
        while (k + 1 < (int) bc_first.size() && f >= bc_first[k + 1]) k++;
        return k;
    };
    P.foff.assign(P.ntiles + 1, 0);
    P.hoff.assign(P.ntiles + 1, 0);
    P.cslot.assign((size_t) P.ntiles * B * P.Wp, (short) -1);
    P.efid.clear();
    P.meta.clear();
    P.halo.clear();
    std::vector<int> fstamp(v.Nf, -1), fentry(v.Nf, 0), hstamp(Nc, -1), hidx(Nc, 0);
    P.Hmax = 0;
    P.Fmax = 0;
    for (int t = 0; t < P.ntiles; t++) {
        const int base = t * B, nb = std::min(B, Nc - base);
        const int h0 = (int) P.halo.size();
        const int e0 = (int) P.efid.size();
        auto local = [&](int ci) -> int {   // ci: internal index
            if (ci >= base && ci < base + nb) return ci - base;
            if (hstamp[ci] != t) {
                hstamp[ci] = t;
                hidx[ci] = (int) P.halo.size() - h0;
                P.halo.push_back(ci);
            }
            return B + hidx[ci];
        };
        for (int c = 0; c < nb; c++) {
            const int ci = base + c, u = perm[ci];
            if (ghost[u]) continue;
            for (int j = cf_off[u], k = 0; j < cf_off[u + 1]; j++, k++) {
                const int f = cf_con[j];
                const int uL = v.fc_con[2 * f], uR = v.fc_con[2 * f + 1];
                if (fstamp[f] != t) {
                    fstamp[f] = t;
                    fentry[f] = (int) P.efid.size() - e0;
                    const int iL = iperm[uL], iR = iperm[uR];
                    const int la = local(iL), lb = local(iR);
                    short m[4] = {(short) la, (short) lb, (short) (f >= F_BC ? bc_of(f) : -1), 0};
                    P.efid.push_back(f);
                    P.meta.insert(P.meta.end(), m, m + 4);
                }
                const int e = fentry[f];
                if (e > 16383) return fail(HCFD_EINVAL, "tile plan: too many faces in one tile");
                P.cslot[((size_t) t * B + c) * P.Wp + k] = (short) ((e << 1) | (uR == u ? 1 : 0));
            }
        }
        if (face_groups) group_entries(P, t, e0, (int) P.efid.size() - e0, nb);
        // pad the entries to a multiple of 4 so every per-tile block is a multiple of 16 B
        while (((int) P.efid.size() - e0) % 4) {
            short m[4] = {0, 0, -1, 0};
            P.efid.push_back(-1);
            P.meta.insert(P.meta.end(), m, m + 4);
        }
        P.foff[t + 1] = (int) P.efid.size();
        P.hoff[t + 1] = (int) P.halo.size();
        P.Hmax = std::max(P.Hmax, (int) P.halo.size() - h0);
        P.Fmax = std::max(P.Fmax, (int) P.efid.size() - e0);
        if (B + P.Hmax > 8191) return fail(HCFD_EINVAL, "tile plan: halo too large");
    }
    return HCFD_OK;
}

}  // namespace hcfd

// ---------------------------------------------------------------------------------------
// Host check of every index the tiled kernels derive from a plan.

extern "C" int hcfd_plan_check(const hcfd_mesh_view* v, int tile, int keep_numbering, long long* info) {
    using namespace hcfd;
    clear_error();
    if (!v) return fail(HCFD_EINVAL, "plan_check: null mesh");
    int rc = validate_view(*v);
    if (rc != HCFD_OK) return rc;
    const int Nc = v->Nc, Nf = v->Nf;
    const int F_BC = v->coloff[v->Ncol - v->NBCcol];
    std::vector<int> cf_off, cf_con;
    build_cf(Nc, Nf, v->fc_con, cf_off, cf_con);
    std::vector<char> ghost(Nc, 0);
    for (int f = F_BC; f < Nf; f++) ghost[v->fc_con[2 * f + 1]] = 1;
    int maxdeg = 0;
    for (int c = 0; c < Nc; c++) if (!ghost[c]) maxdeg = std::max(maxdeg, cf_off[c + 1] - cf_off[c]);
    const int W = maxdeg <= 3 ? 3 : maxdeg <= 4 ? 4 : 8;
    std::vector<int> perm;
    if (keep_numbering) { perm.resize(Nc); std::iota(perm.begin(), perm.end(), 0); }
    else perm = morton_order(*v);
    std::vector<int> bc_first;
    for (int col = v->Ncol - v->NBCcol; col < v->Ncol; col++) bc_first.push_back(v->coloff[col]);
    const int B = tile ? tile : 256;
    std::vector<int> iperm(Nc);
    // both entry orders: as the cells meet their faces (pass 1, the arena) and grouped for
    // pass 2's face phase; info describes the first
    for (int grouped = 1; grouped >= 0; grouped--) {
    TilePlan P;
    rc = build_tile_plan(*v, cf_off, cf_con, ghost, perm, F_BC, bc_first, B, W, P, grouped != 0);
    if (rc != HCFD_OK) return rc;
    for (int i = 0; i < Nc; i++) iperm[perm[i]] = i;
    auto bad = [&](const char* what, int t) {
        return fail(HCFD_EINVAL, std::string("plan_check: ") + what + " (tile " + std::to_string(t) + ")");
    };
    const int E = (int) P.efid.size();
    if (P.foff[0] != 0 || P.foff[P.ntiles] != E || P.hoff[0] != 0 || P.hoff[P.ntiles] != (int) P.halo.size())
        return bad("offset arrays do not span", -1);
    long long cut = 0, internal = 0;
    std::vector<int> seen(2 * (size_t) P.Fmax);
    for (int t = 0; t < P.ntiles; t++) {
        const int base = t * B, nb = std::min(B, Nc - base);
        const int f0 = P.foff[t], nf = P.foff[t + 1] - f0, h0 = P.hoff[t], nh = P.hoff[t + 1] - h0;
        if (nf < 0 || nh < 0 || nf % 4 || nf > P.Fmax || nh > P.Hmax) return bad("entry or halo count", t);
        // bulk-copy sizes and offsets: multiples of 16 bytes (float and double layouts)
        if ((f0 * 8) % 16 || (base * P.Wp * 2) % 16 || (B * P.Wp * 2) % 16) return bad("bulk alignment", t);
        for (int h = 0; h < nh; h++) {
            const int ci = P.halo[h0 + h];
            if (ci < 0 || ci >= Nc || (ci >= base && ci < base + nb)) return bad("halo id", t);
        }
        auto cell_of = [&](int l) { return l < B ? base + l : P.halo[h0 + l - B]; };
        std::fill(seen.begin(), seen.end(), 0);
        for (int e = 0; e < nf; e++) {
            const short* m = &P.meta[4 * (size_t) (f0 + e)];
            const int la = m[0], lb = m[1], bc = m[2];
            const int f = P.efid[f0 + e];
            const bool okl = (la < nb) || (la >= B && la < B + nh);
            const bool okr = (lb < nb) || (lb >= B && lb < B + nh);
            if (la < 0 || lb < 0 || !okl || !okr) return bad("local cell index", t);
            if (f < 0) {
                if (bc != -1) return bad("padding entry with a boundary index", t);
                continue;
            }
            if (cell_of(la) != iperm[v->fc_con[2 * f]] || cell_of(lb) != iperm[v->fc_con[2 * f + 1]])
                return bad("entry cells differ from the face's cells", t);
            if ((f >= F_BC) != (bc >= 0) || bc >= (int) bc_first.size()) return bad("boundary index", t);
            const bool inL = la < B && !ghost[perm[base + la]], inR = lb < B && !ghost[perm[base + lb]];
            if (inL && inR) internal++; else cut++;
        }
        // every real tile cell lists exactly its faces, in increasing face order, each entry
        // on the side the entry records; every side of an entry is listed by its tile cell
        for (int c = 0; c < nb; c++) {
            const int u = perm[base + c];
            const short* cs = &P.cslot[((size_t) t * B + c) * P.Wp];
            const int deg = ghost[u] ? 0 : cf_off[u + 1] - cf_off[u];
            for (int k = 0; k < P.Wp; k++) {
                if (k >= deg) {
                    if (cs[k] != -1) return bad("slot beyond the cell's faces", t);
                    continue;
                }
                if (cs[k] < 0) return bad("missing slot", t);
                const int e = cs[k] >> 1, side = cs[k] & 1;
                if (e >= nf) return bad("slot entry out of range", t);
                const short* m = &P.meta[4 * (size_t) (f0 + e)];
                if ((side ? m[1] : m[0]) != c) return bad("slot side", t);
                if (P.efid[f0 + e] != cf_con[cf_off[u] + k]) return bad("slot face order", t);
                if (seen[2 * e + side]++) return bad("entry side listed twice", t);
            }
        }
        for (int e = 0; e < nf; e++) {
            const short* m = &P.meta[4 * (size_t) (f0 + e)];
            if (P.efid[f0 + e] < 0) continue;
            for (int side = 0; side < 2; side++) {
                const int l = m[side];
                const bool real_in_tile = l < nb && !ghost[perm[base + l]];
                if (real_in_tile != (seen[2 * e + side] == 1)) return bad("entry side not listed by its cell", t);
            }
        }
    }
    if (info && !grouped) {
        info[0] = P.ntiles; info[1] = P.Hmax; info[2] = P.Fmax; info[3] = E;
        info[4] = internal; info[5] = cut; info[6] = W; info[7] = (long long) P.halo.size();
    }
    }
    return HCFD_OK;
}
