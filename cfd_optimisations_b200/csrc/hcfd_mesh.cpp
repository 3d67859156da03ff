// Host mesh handling for the B200 solver: the .hmsh reader and writer, mesh validation,
// the cell->face table, the supersonic-wedge generator and cell renumbering.
//
// File layout (.hmsh): the reference's reader is src/Mesh.cpp:7-54 and its writer
// interface/Mesh.py:441-463.  Face ordering conventions follow interface/Mesh.py:321-378.
#include "hcfd_internal.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <queue>

namespace hcfd {

static thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}
void clear_error() { g_err.clear(); }

void build_cf(int Nc, int Nf, const int* fc_con, std::vector<int>& cf_off, std::vector<int>& cf_con) {
    // Mesh::compute_cf_con (src/Mesh.cpp:88-117): counts, prefix sum, then a pass over the
    // faces in increasing index so each cell's list is sorted by face.
    cf_off.assign(Nc + 1, 0);
    for (int f = 0; f < Nf; f++) {
        cf_off[fc_con[2 * f] + 1]++;
        cf_off[fc_con[2 * f + 1] + 1]++;
    }
    for (int i = 0; i < Nc; i++) cf_off[i + 1] += cf_off[i];
    cf_con.assign(cf_off[Nc], 0);
    std::vector<int> cnt(Nc, 0);
    for (int f = 0; f < Nf; f++) {
        int L = fc_con[2 * f], R = fc_con[2 * f + 1];
        cf_con[cf_off[L] + cnt[L]++] = f;
        cf_con[cf_off[R] + cnt[R]++] = f;
    }
}

int validate_view(const hcfd_mesh_view& v) {
    if (v.dim != 2) return fail(HCFD_EINVAL, "mesh: only dim == 2 is supported");
    if (v.Nn <= 0 || v.Nc <= 0 || v.Nf <= 0 || v.Ncol <= 0 || v.NBCcol < 0 || v.NBCcol > v.Ncol)
        return fail(HCFD_EINVAL, "mesh: bad counts");
    if (!v.coltag || !v.coloff || !v.nodes || !v.fn_con || !v.fc_con || !v.cn_off || !v.cn_con)
        return fail(HCFD_EINVAL, "mesh: null array");
    if (v.coloff[0] != 0 || v.coloff[v.Ncol] != v.Nf) return fail(HCFD_EINVAL, "mesh: coloff does not span the faces");
    for (int c = 0; c < v.Ncol; c++)
        if (v.coloff[c + 1] < v.coloff[c]) return fail(HCFD_EINVAL, "mesh: coloff not monotone");
    if (v.cn_off[0] != 0) return fail(HCFD_EINVAL, "mesh: cn_off[0] != 0");
    for (int i = 0; i < v.Nc; i++)
        if (v.cn_off[i + 1] <= v.cn_off[i]) return fail(HCFD_EINVAL, "mesh: cell without nodes");
    const int ncn = v.cn_off[v.Nc];
    for (int k = 0; k < ncn; k++)
        if (v.cn_con[k] < 0 || v.cn_con[k] >= v.Nn) return fail(HCFD_EINVAL, "mesh: cn_con out of range");
    for (int f = 0; f < v.Nf; f++) {
        int a = v.fn_con[2 * f], b = v.fn_con[2 * f + 1];
        int L = v.fc_con[2 * f], R = v.fc_con[2 * f + 1];
        if (a < 0 || a >= v.Nn || b < 0 || b >= v.Nn || a == b) return fail(HCFD_EINVAL, "mesh: fn_con out of range");
        if (L < 0 || L >= v.Nc || R < 0 || R >= v.Nc || L == R) return fail(HCFD_EINVAL, "mesh: fc_con out of range");
    }
    // Ghost conventions the step relies on (interface/Mesh.py:336-338): every boundary
    // face's right cell is a ghost with that face as its only face, and no ghost appears
    // on an interior face or on the left of a face.
    const int F_BC = v.coloff[v.Ncol - v.NBCcol];
    std::vector<int> deg(v.Nc, 0), ghost(v.Nc, 0);
    for (int f = 0; f < v.Nf; f++) { deg[v.fc_con[2 * f]]++; deg[v.fc_con[2 * f + 1]]++; }
    for (int f = F_BC; f < v.Nf; f++) ghost[v.fc_con[2 * f + 1]] = 1;
    for (int f = 0; f < v.Nf; f++) {
        int L = v.fc_con[2 * f], R = v.fc_con[2 * f + 1];
        if (ghost[L]) return fail(HCFD_EINVAL, "mesh: ghost cell on the left of a face");
        if (f < F_BC && ghost[R]) return fail(HCFD_EINVAL, "mesh: ghost cell on an interior face");
        if (f >= F_BC && deg[R] != 1) return fail(HCFD_EINVAL, "mesh: ghost cell with more than one face");
    }
    for (int i = 0; i < v.Nc; i++)
        if (deg[i] == 0) return fail(HCFD_EINVAL, "mesh: cell without faces");
    return HCFD_OK;
}

}  // namespace hcfd

using hcfd::fail;

namespace {

hcfd_mesh_view view_of(const hcfd_mesh& m) {
    hcfd_mesh_view v;
    v.dim = m.dim; v.Nn = m.Nn; v.Ncol = m.Ncol; v.NBCcol = m.NBCcol; v.Nc = m.Nc; v.Nf = m.Nf;
    v.coltag = m.coltag.data(); v.coloff = m.coloff.data(); v.nodes = m.nodes.data();
    v.fn_con = m.fn_con.data(); v.fc_con = m.fc_con.data();
    v.cn_off = m.cn_off.data(); v.cn_con = m.cn_con.data();
    v.cc_off = m.cc_off.empty() ? nullptr : m.cc_off.data();
    v.cc_con = m.cc_off.empty() ? nullptr : m.cc_con.data();
    return v;
}

// Neighbour lists from the faces, each sorted ascending (the cc table of
// interface/Mesh.py:283-294: cells sharing a face).
void build_cc(hcfd_mesh& m) {
    m.cc_off.assign(m.Nc + 1, 0);
    for (int f = 0; f < m.Nf; f++) { m.cc_off[m.fc_con[2 * f] + 1]++; m.cc_off[m.fc_con[2 * f + 1] + 1]++; }
    for (int i = 0; i < m.Nc; i++) m.cc_off[i + 1] += m.cc_off[i];
    m.cc_con.assign(m.cc_off[m.Nc], 0);
    std::vector<int> cnt(m.Nc, 0);
    for (int f = 0; f < m.Nf; f++) {
        int L = m.fc_con[2 * f], R = m.fc_con[2 * f + 1];
        m.cc_con[m.cc_off[L] + cnt[L]++] = R;
        m.cc_con[m.cc_off[R] + cnt[R]++] = L;
    }
    for (int i = 0; i < m.Nc; i++) std::sort(m.cc_con.begin() + m.cc_off[i], m.cc_con.begin() + m.cc_off[i + 1]);
}

// Faces inside each colour sorted by (min cell, max cell); interior faces oriented
// CL < CR; boundary faces keep the ghost (already on the right) on the right.  This is
// the order interface/Mesh.py:321-378 produces from the COO order of the cc matrix.
void sort_faces(hcfd_mesh& m) {
    const int F_BC = m.coloff[m.Ncol - m.NBCcol];
    std::vector<int> ord(m.Nf);
    std::vector<unsigned long long> key(m.Nf);
    for (int f = 0; f < m.Nf; f++) {
        int L = m.fc_con[2 * f], R = m.fc_con[2 * f + 1];
        if (f < F_BC && L > R) { std::swap(L, R); std::swap(m.fc_con[2 * f], m.fc_con[2 * f + 1]); }
        unsigned lo = (unsigned) std::min(L, R), hi = (unsigned) std::max(L, R);
        key[f] = ((unsigned long long) lo << 32) | hi;
    }
    for (int c = 0; c < m.Ncol; c++) {
        int a = m.coloff[c], b = m.coloff[c + 1];
        std::iota(ord.begin() + a, ord.begin() + b, a);
        std::sort(ord.begin() + a, ord.begin() + b, [&](int x, int y) { return key[x] < key[y]; });
    }
    std::vector<int> fc(2 * m.Nf), fn(2 * m.Nf);
    for (int k = 0; k < m.Nf; k++) {
        int f = ord[k];
        fc[2 * k] = m.fc_con[2 * f]; fc[2 * k + 1] = m.fc_con[2 * f + 1];
        fn[2 * k] = m.fn_con[2 * f]; fn[2 * k + 1] = m.fn_con[2 * f + 1];
    }
    m.fc_con.swap(fc);
    m.fn_con.swap(fn);
}

// perm[new] = old.
void apply_cell_perm(hcfd_mesh& m, const std::vector<int>& perm) {
    std::vector<int> inv(m.Nc);
    for (int i = 0; i < m.Nc; i++) inv[perm[i]] = i;
    std::vector<int> cn_off(m.Nc + 1, 0), cn_con, ct(m.Nc, 0);
    cn_con.reserve(m.cn_con.size());
    for (int i = 0; i < m.Nc; i++) {
        int o = perm[i];
        for (int k = m.cn_off[o]; k < m.cn_off[o + 1]; k++) cn_con.push_back(m.cn_con[k]);
        cn_off[i + 1] = (int) cn_con.size();
        if (!m.c_ctypes.empty()) ct[i] = m.c_ctypes[o];
    }
    m.cn_off.swap(cn_off);
    m.cn_con.swap(cn_con);
    if (!m.c_ctypes.empty()) m.c_ctypes.swap(ct);
    for (int k = 0; k < 2 * m.Nf; k++) m.fc_con[k] = inv[m.fc_con[k]];
    sort_faces(m);
    build_cc(m);
    hcfd::build_cf(m.Nc, m.Nf, m.fc_con.data(), m.cf_off, m.cf_con);
}

struct SplitMix {
    unsigned long long s;
    explicit SplitMix(unsigned long long seed) : s(seed) {}
    unsigned long long next() {
        unsigned long long z = (s += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }  // [0, 1)
};

std::vector<int> random_perm(int n, unsigned long long seed) {
    std::vector<int> p(n);
    std::iota(p.begin(), p.end(), 0);
    SplitMix r(seed ^ 0xA5A5A5A5DEADBEEFULL);
    for (int i = n - 1; i > 0; i--) {
        int j = (int) (r.next() % (unsigned long long) (i + 1));
        std::swap(p[i], p[j]);
    }
    return p;
}

// Reverse Cuthill-McKee over the face adjacency: per connected component, a BFS from a
// pseudo-peripheral cell (repeated BFS from the minimum-degree cell of the last level),
// neighbours visited in increasing degree, and the final order reversed.
std::vector<int> rcm_perm(const hcfd_mesh& m) {
    const int n = m.Nc;
    std::vector<int> deg(n);
    for (int i = 0; i < n; i++) deg[i] = m.cc_off[i + 1] - m.cc_off[i];
    std::vector<int> order;
    order.reserve(n);
    std::vector<char> seen(n, 0);
    std::vector<int> level(n, -1), nb;
    auto bfs_last = [&](int s, std::vector<int>& touched) {
        // BFS from s over unseen cells; returns a minimum-degree cell of the last level.
        touched.clear();
        std::queue<int> q;
        q.push(s); level[s] = 0; touched.push_back(s);
        int maxl = 0;
        while (!q.empty()) {
            int c = q.front(); q.pop();
            for (int k = m.cc_off[c]; k < m.cc_off[c + 1]; k++) {
                int d = m.cc_con[k];
                if (seen[d] || level[d] >= 0) continue;
                level[d] = level[c] + 1;
                maxl = std::max(maxl, level[d]);
                touched.push_back(d);
                q.push(d);
            }
        }
        int best = -1;
        for (int c : touched) if (level[c] == maxl && (best < 0 || deg[c] < deg[best])) best = c;
        for (int c : touched) level[c] = -1;
        return best;
    };
    std::vector<int> touched;
    std::vector<int> bydeg(n);
    std::iota(bydeg.begin(), bydeg.end(), 0);
    std::stable_sort(bydeg.begin(), bydeg.end(), [&](int a, int b) { return deg[a] < deg[b]; });
    for (int start0 : bydeg) {
        if (seen[start0]) continue;
        int s = start0;
        for (int it = 0; it < 3; it++) { int t = bfs_last(s, touched); if (t == s) break; s = t; }
        std::queue<int> q;
        q.push(s); seen[s] = 1;
        while (!q.empty()) {
            int c = q.front(); q.pop();
            order.push_back(c);
            nb.clear();
            for (int k = m.cc_off[c]; k < m.cc_off[c + 1]; k++) if (!seen[m.cc_con[k]]) nb.push_back(m.cc_con[k]);
            std::sort(nb.begin(), nb.end(), [&](int a, int b) { return deg[a] != deg[b] ? deg[a] < deg[b] : a < b; });
            for (int d : nb) { seen[d] = 1; q.push(d); }
        }
    }
    std::reverse(order.begin(), order.end());
    return order;
}

unsigned long long spread32(unsigned long long x) {
    x &= 0xFFFFFFFFULL;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFULL;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFULL;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0FULL;
    x = (x | (x << 2)) & 0x3333333333333333ULL;
    x = (x | (x << 1)) & 0x5555555555555555ULL;
    return x;
}

// Cells sorted by the Morton (Z-order) key of their vertex-average centre, quantised to
// 2^31 steps over the node bounding box.
std::vector<int> morton_perm(const hcfd_mesh& m) {
    double lo[2] = {1e300, 1e300}, hi[2] = {-1e300, -1e300};
    for (int i = 0; i < m.Nn; i++)
        for (int d = 0; d < 2; d++) { lo[d] = std::min(lo[d], m.nodes[2 * i + d]); hi[d] = std::max(hi[d], m.nodes[2 * i + d]); }
    std::vector<unsigned long long> key(m.Nc);
    for (int c = 0; c < m.Nc; c++) {
        double x[2] = {0, 0};
        int nn = m.cn_off[c + 1] - m.cn_off[c];
        for (int k = m.cn_off[c]; k < m.cn_off[c + 1]; k++)
            for (int d = 0; d < 2; d++) x[d] += m.nodes[2 * m.cn_con[k] + d] / nn;
        unsigned long long q[2];
        for (int d = 0; d < 2; d++) {
            double t = (hi[d] > lo[d]) ? (x[d] - lo[d]) / (hi[d] - lo[d]) : 0.0;
            t = std::min(std::max(t, 0.0), 1.0);
            q[d] = (unsigned long long) (t * 2147483647.0);
        }
        key[c] = spread32(q[0]) | (spread32(q[1]) << 1);
    }
    std::vector<int> p(m.Nc);
    std::iota(p.begin(), p.end(), 0);
    std::stable_sort(p.begin(), p.end(), [&](int a, int b) { return key[a] < key[b]; });
    return p;
}

int renumber(hcfd_mesh& m, int numbering, unsigned long long seed) {
    switch (numbering) {
    case HCFD_NUMBER_NATURAL: return HCFD_OK;
    case HCFD_NUMBER_RANDOM: apply_cell_perm(m, random_perm(m.Nc, seed)); return HCFD_OK;
    case HCFD_NUMBER_RCM:
        if (m.cc_off.empty()) build_cc(m);
        apply_cell_perm(m, rcm_perm(m));
        return HCFD_OK;
    case HCFD_NUMBER_MORTON: apply_cell_perm(m, morton_perm(m)); return HCFD_OK;
    default: return fail(HCFD_EINVAL, "renumber: unknown numbering");
    }
}

// Faces from cell-node connectivity: cells sharing an edge (two nodes) are neighbours,
// the rule interface/Mesh.py:283-294 applies (cn cn^T >= dim).  Each edge must belong to
// exactly two cells.  A face's colour is the larger colour tag of its two cells
// (interface/Mesh.py:331-334); cells of tag > 0 are ghosts and go on the right.
int build_faces(hcfd_mesh& m, const std::vector<int>& ctag, int ntags) {
    struct E { unsigned long long key; int cell; };
    std::vector<E> e;
    e.reserve(m.cn_con.size());
    for (int c = 0; c < m.Nc; c++) {
        int a = m.cn_off[c], n = m.cn_off[c + 1] - a;
        if (n == 2) {
            int u = m.cn_con[a], v = m.cn_con[a + 1];
            e.push_back({((unsigned long long) std::min(u, v) << 32) | (unsigned) std::max(u, v), c});
        } else {
            for (int k = 0; k < n; k++) {
                int u = m.cn_con[a + k], v = m.cn_con[a + (k + 1) % n];
                e.push_back({((unsigned long long) std::min(u, v) << 32) | (unsigned) std::max(u, v), c});
            }
        }
    }
    std::sort(e.begin(), e.end(), [](const E& x, const E& y) { return x.key != y.key ? x.key < y.key : x.cell < y.cell; });
    std::vector<std::vector<int>> byc(ntags);
    std::vector<int> fc, fn;
    for (size_t i = 0; i < e.size();) {
        size_t j = i;
        while (j < e.size() && e[j].key == e[i].key) j++;
        if (j - i != 2) return fail(HCFD_EINVAL, "mesh: an edge is not shared by exactly two cells");
        int c1 = e[i].cell, c2 = e[i + 1].cell;
        int col = std::max(ctag[c1], ctag[c2]);
        if (ctag[c1] > 0 && ctag[c2] > 0) return fail(HCFD_EINVAL, "mesh: two ghost cells share an edge");
        int L = c1, R = c2;
        if (ctag[L] > ctag[R] || (col == 0 && L > R)) std::swap(L, R);
        byc[col].push_back((int) (fc.size() / 2));
        fc.push_back(L); fc.push_back(R);
        fn.push_back((int) (e[i].key >> 32)); fn.push_back((int) (e[i].key & 0xFFFFFFFFULL));
        i = j;
    }
    m.Nf = (int) (fc.size() / 2);
    m.Ncol = ntags;
    m.coltag.resize(ntags);
    m.coloff.assign(ntags + 1, 0);
    m.fc_con.resize(2 * m.Nf);
    m.fn_con.resize(2 * m.Nf);
    int k = 0;
    for (int c = 0; c < ntags; c++) {
        m.coltag[c] = c;
        for (int f : byc[c]) {
            m.fc_con[2 * k] = fc[2 * f]; m.fc_con[2 * k + 1] = fc[2 * f + 1];
            m.fn_con[2 * k] = fn[2 * f]; m.fn_con[2 * k + 1] = fn[2 * f + 1];
            k++;
        }
        m.coloff[c + 1] = k;
    }
    sort_faces(m);
    build_cc(m);
    hcfd::build_cf(m.Nc, m.Nf, m.fc_con.data(), m.cf_off, m.cf_con);
    return HCFD_OK;
}

}  // namespace

extern "C" {

int hcfd_mesh_load(const char* path, hcfd_mesh** out) {
    hcfd::clear_error();
    if (!path || !out) return fail(HCFD_EINVAL, "mesh_load: null argument");
    *out = nullptr;
    FILE* fp = fopen(path, "rb");
    if (!fp) return fail(HCFD_EIO, std::string("mesh_load: cannot open ") + path);
    std::vector<char> buf;
    {
        fseek(fp, 0, SEEK_END);
        long sz = ftell(fp);
        fseek(fp, 0, SEEK_SET);
        if (sz < 32) { fclose(fp); return fail(HCFD_EIO, "mesh_load: file shorter than its header"); }
        buf.resize((size_t) sz);
        size_t got = fread(buf.data(), 1, (size_t) sz, fp);
        fclose(fp);
        if (got != (size_t) sz) return fail(HCFD_EIO, "mesh_load: short read");
    }
    size_t off = 0;
    auto take = [&](void* dst, size_t bytes) -> bool {
        if (off + bytes > buf.size()) return false;
        if (bytes) std::memcpy(dst, buf.data() + off, bytes);
        off += bytes;
        return true;
    };
    int N[8];
    take(N, sizeof(N));
    auto* m = new hcfd_mesh();
    // src/Mesh.cpp:13-21
    m->dim = N[0]; m->Nn = N[1]; m->Ncol = N[2]; m->NBCcol = N[3]; m->Nc = N[4]; m->Nf = N[5];
    const int npn = std::max(1, N[6]), nch = N[7];
    if (m->dim != 2 || m->Nn <= 0 || m->Ncol <= 0 || m->NBCcol < 0 || m->NBCcol > m->Ncol || m->Nc <= 0 ||
        m->Nf <= 0 || nch < 0) {
        delete m;
        return fail(HCFD_EINVAL, "mesh_load: bad header");
    }
    std::vector<char> names((size_t) nch);
    bool ok = take(names.data(), (size_t) nch);
    m->coltag.resize(m->Ncol); m->coloff.resize(m->Ncol + 1);
    m->nodes.resize((size_t) m->Nn * 2);
    m->fn_con.resize((size_t) 2 * m->Nf); m->fc_con.resize((size_t) 2 * m->Nf);
    m->cn_off.resize(m->Nc + 1); m->cc_off.resize(m->Nc + 1);
    ok = ok && take(m->coltag.data(), 4 * m->coltag.size()) && take(m->coloff.data(), 4 * m->coloff.size()) &&
         take(m->nodes.data(), 8 * m->nodes.size()) && take(m->fn_con.data(), 4 * m->fn_con.size()) &&
         take(m->fc_con.data(), 4 * m->fc_con.size()) && take(m->cn_off.data(), 4 * m->cn_off.size());
    if (ok && (m->cn_off[m->Nc] < 0 || (size_t) m->cn_off[m->Nc] * 4 > buf.size())) ok = false;
    if (ok) { m->cn_con.resize(m->cn_off[m->Nc]); ok = take(m->cn_con.data(), 4 * m->cn_con.size()); }
    ok = ok && take(m->cc_off.data(), 4 * m->cc_off.size());
    if (ok && (m->cc_off[m->Nc] < 0 || (size_t) m->cc_off[m->Nc] * 4 > buf.size())) ok = false;
    if (ok) { m->cc_con.resize(m->cc_off[m->Nc]); ok = take(m->cc_con.data(), 4 * m->cc_con.size()); }
    if (!ok) { delete m; return fail(HCFD_EIO, "mesh_load: truncated file"); }
    if (off + 4 * (size_t) m->Nc <= buf.size()) { m->c_ctypes.resize(m->Nc); take(m->c_ctypes.data(), 4 * m->Nc); }
    // Mesh::parse_pnames (src/Mesh.cpp:70-86): npn NUL-terminated strings.
    size_t p = 0;
    for (int k = 0; k < npn && p <= names.size(); k++) {
        size_t q = p;
        while (q < names.size() && names[q] != '\0') q++;
        m->pnames.emplace_back(names.data() + p, q - p);
        p = q + 1;
    }
    hcfd_mesh_view v = view_of(*m);
    v.cc_off = nullptr; v.cc_con = nullptr;
    int rc = hcfd::validate_view(v);
    if (rc != HCFD_OK) { delete m; return rc; }
    hcfd::build_cf(m->Nc, m->Nf, m->fc_con.data(), m->cf_off, m->cf_con);
    *out = m;
    return HCFD_OK;
}

int hcfd_mesh_write(const hcfd_mesh* m, const char* path) {
    hcfd::clear_error();
    if (!m || !path) return fail(HCFD_EINVAL, "mesh_write: null argument");
    FILE* fp = fopen(path, "wb");
    if (!fp) return fail(HCFD_EIO, std::string("mesh_write: cannot open ") + path);
    std::string names;
    for (const auto& s : m->pnames) { names += s; names.push_back('\0'); }
    int N[8] = {m->dim, m->Nn, m->Ncol, m->NBCcol, m->Nc, m->Nf, (int) m->pnames.size(), (int) names.size()};
    std::vector<int> cc_off = m->cc_off, cc_con = m->cc_con, ct = m->c_ctypes;
    if (cc_off.empty()) {
        hcfd_mesh tmp = *m;
        build_cc(tmp);
        cc_off = tmp.cc_off; cc_con = tmp.cc_con;
    }
    if (ct.empty()) {
        ct.resize(m->Nc);
        for (int i = 0; i < m->Nc; i++) {
            int n = m->cn_off[i + 1] - m->cn_off[i];
            ct[i] = n == 2 ? 1 : n == 3 ? 2 : n == 4 ? 3 : 0;   // gmsh element types
        }
    }
    bool ok = fwrite(N, 4, 8, fp) == 8;
    auto put = [&](const void* p, size_t sz, size_t n) { if (n) ok = ok && fwrite(p, sz, n, fp) == n; };
    put(names.data(), 1, names.size());
    put(m->coltag.data(), 4, m->coltag.size());
    put(m->coloff.data(), 4, m->coloff.size());
    put(m->nodes.data(), 8, m->nodes.size());
    put(m->fn_con.data(), 4, m->fn_con.size());
    put(m->fc_con.data(), 4, m->fc_con.size());
    put(m->cn_off.data(), 4, m->cn_off.size());
    put(m->cn_con.data(), 4, m->cn_con.size());
    put(cc_off.data(), 4, cc_off.size());
    put(cc_con.data(), 4, cc_con.size());
    put(ct.data(), 4, ct.size());
    ok = (fclose(fp) == 0) && ok;
    return ok ? HCFD_OK : fail(HCFD_EIO, "mesh_write: write failed");
}

int hcfd_mesh_view_of(const hcfd_mesh* m, hcfd_mesh_view* v) {
    if (!m || !v) return fail(HCFD_EINVAL, "mesh_view_of: null argument");
    *v = view_of(*m);
    return HCFD_OK;
}

int hcfd_mesh_cf(const hcfd_mesh* m, const int** cf_off, const int** cf_con) {
    if (!m || !cf_off || !cf_con) return fail(HCFD_EINVAL, "mesh_cf: null argument");
    *cf_off = m->cf_off.data();
    *cf_con = m->cf_con.data();
    return HCFD_OK;
}

const char* hcfd_mesh_pname(const hcfd_mesh* m, int k) {
    if (!m || k < 0 || k >= (int) m->pnames.size()) return nullptr;
    return m->pnames[k].c_str();
}

void hcfd_mesh_free(hcfd_mesh* m) { delete m; }

int hcfd_mesh_renumber(hcfd_mesh* m, int numbering, uint64_t seed) {
    hcfd::clear_error();
    if (!m) return fail(HCFD_EINVAL, "mesh_renumber: null mesh");
    return renumber(*m, numbering, seed);
}

int hcfd_mesh_generate_wedge(const hcfd_wedge_spec* sp, hcfd_mesh** out) {
    hcfd::clear_error();
    if (!sp || !out) return fail(HCFD_EINVAL, "generate_wedge: null argument");
    *out = nullptr;
    const int nx = sp->nx, ny = sp->ny;
    if (nx < 3 || ny < 3 || (long long) nx * ny > (1LL << 29)) return fail(HCFD_EINVAL, "generate_wedge: bad node grid");
    if (!(sp->length > 0) || !(sp->height > 0) || !(sp->jitter >= 0 && sp->jitter < 0.5) ||
        !(sp->theta_deg >= 0 && sp->theta_deg < 60))
        return fail(HCFD_EINVAL, "generate_wedge: bad geometry");
    auto* m = new hcfd_mesh();
    m->dim = 2;
    m->Nn = nx * ny;
    m->nodes.resize((size_t) 2 * m->Nn);
    const double tanth = std::tan(sp->theta_deg * M_PI / 180.0);
    const double hx = sp->length / (nx - 1);
    SplitMix rng(sp->seed);
    for (int j = 0; j < ny; j++) {
        for (int i = 0; i < nx; i++) {
            double x = sp->length * i / (nx - 1);
            double yb = std::max(0.0, (x - sp->x_ramp) * tanth);
            if (yb >= sp->height) { delete m; return fail(HCFD_EINVAL, "generate_wedge: ramp reaches the top wall"); }
            double y = yb + (sp->height - yb) * j / (ny - 1);
            if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && sp->jitter > 0) {
                double hy = (sp->height - yb) / (ny - 1);
                x += (2.0 * rng.uniform() - 1.0) * sp->jitter * hx;
                y += (2.0 * rng.uniform() - 1.0) * sp->jitter * hy;
            }
            m->nodes[2 * (j * nx + i)] = x;
            m->nodes[2 * (j * nx + i) + 1] = y;
        }
    }
    const int ntri = 2 * (nx - 1) * (ny - 1), ng = 2 * (nx - 1) + 2 * (ny - 1);
    m->Nc = ntri + ng;
    m->cn_off.resize(m->Nc + 1);
    m->cn_con.reserve((size_t) 3 * ntri + 2 * ng);
    m->c_ctypes.resize(m->Nc);
    std::vector<int> ctag(m->Nc, 0);
    int c = 0;
    m->cn_off[0] = 0;
    auto push = [&](std::initializer_list<int> nds, int tag) {
        for (int n : nds) m->cn_con.push_back(n);
        ctag[c] = tag;
        m->c_ctypes[c] = nds.size() == 2 ? 1 : 2;
        m->cn_off[++c] = (int) m->cn_con.size();
    };
    auto N = [&](int i, int j) { return j * nx + i; };
    for (int j = 0; j < ny - 1; j++) {
        for (int i = 0; i < nx - 1; i++) {
            int a = N(i, j), b = N(i + 1, j), cc = N(i + 1, j + 1), d = N(i, j + 1);
            if (rng.next() >> 63) { push({a, b, cc}, 0); push({a, cc, d}, 0); }
            else                  { push({a, b, d}, 0);  push({b, cc, d}, 0); }
        }
    }
    for (int i = 0; i < nx - 1; i++) push({N(i, ny - 1), N(i + 1, ny - 1)}, 1);   // upper
    for (int i = 0; i < nx - 1; i++) push({N(i, 0), N(i + 1, 0)}, 2);             // lower
    for (int j = 0; j < ny - 1; j++) push({N(0, j), N(0, j + 1)}, 3);             // inlet
    for (int j = 0; j < ny - 1; j++) push({N(nx - 1, j), N(nx - 1, j + 1)}, 4);   // outlet
    // Every triangle must keep a positive area after the jitter.
    for (int t = 0; t < ntri; t++) {
        const int* n3 = &m->cn_con[m->cn_off[t]];
        double ax = m->nodes[2 * n3[0]], ay = m->nodes[2 * n3[0] + 1];
        double bx = m->nodes[2 * n3[1]], by = m->nodes[2 * n3[1] + 1];
        double cx = m->nodes[2 * n3[2]], cy = m->nodes[2 * n3[2] + 1];
        if ((bx - ax) * (cy - ay) - (by - ay) * (cx - ax) <= 0) {
            delete m;
            return fail(HCFD_EINVAL, "generate_wedge: a triangle is inverted (jitter too large)");
        }
    }
    m->NBCcol = 4;
    m->pnames = {"upper", "lower", "inlet", "outlet"};
    int rc = build_faces(*m, ctag, 5);
    if (rc == HCFD_OK) rc = renumber(*m, sp->numbering, sp->seed);
    if (rc != HCFD_OK) { delete m; return rc; }
    *out = m;
    return HCFD_OK;
}

int hcfd_write_hsln(const char* path, int nvars, const char* const* varnames, int Nc, const double* const* arrs) {
    // Writer::write_soln (src/Writer.cpp:22-39).
    hcfd::clear_error();
    if (!path || nvars <= 0 || Nc <= 0 || !varnames || !arrs) return fail(HCFD_EINVAL, "write_hsln: bad argument");
    int nchars = 0;
    for (int v = 0; v < nvars; v++) nchars += (int) std::strlen(varnames[v]) + 1;
    FILE* fp = fopen(path, "wb");
    if (!fp) return fail(HCFD_EIO, std::string("write_hsln: cannot open ") + path);
    bool ok = fwrite(&Nc, 4, 1, fp) == 1 && fwrite(&nvars, 4, 1, fp) == 1 && fwrite(&nchars, 4, 1, fp) == 1;
    for (int v = 0; v < nvars && ok; v++) {
        size_t n = std::strlen(varnames[v]) + 1;
        ok = fwrite(varnames[v], 1, n, fp) == n;
    }
    for (int v = 0; v < nvars && ok; v++) ok = fwrite(arrs[v], 8, (size_t) Nc, fp) == (size_t) Nc;
    ok = (fclose(fp) == 0) && ok;
    return ok ? HCFD_OK : fail(HCFD_EIO, "write_hsln: write failed");
}

int hcfd_checkpoint_info(const char* path, int* Nc, int* precision, long long* steps, int* has_limiter) {
    hcfd::clear_error();
    if (!path) return fail(HCFD_EINVAL, "checkpoint_info: null path");
    hcfd::CkptHeader h;
    int rc = hcfd::ckpt_read(path, h, nullptr, nullptr);
    if (rc) return rc;
    if (Nc) *Nc = h.Nc;
    if (precision) *precision = h.precision;
    if (steps) *steps = h.steps;
    if (has_limiter) *has_limiter = h.has_phiF;
    return HCFD_OK;
}

const char* hcfd_last_error(void) { return hcfd::g_err.c_str(); }

}  // extern "C"

namespace hcfd {

int ckpt_write(const char* path, const CkptHeader& h, const std::vector<double>& U, const std::vector<double>* phiF) {
    if (!path) return fail(HCFD_EINVAL, "checkpoint: null path");
    FILE* fp = fopen(path, "wb");
    if (!fp) return fail(HCFD_EIO, std::string("checkpoint: cannot open ") + path);
    bool ok = fwrite(&h, sizeof(h), 1, fp) == 1 && fwrite(U.data(), 8, U.size(), fp) == U.size();
    if (ok && phiF) ok = fwrite(phiF->data(), 8, phiF->size(), fp) == phiF->size();
    ok = (fclose(fp) == 0) && ok;
    return ok ? HCFD_OK : fail(HCFD_EIO, std::string("checkpoint: write failed: ") + path);
}

int ckpt_read(const char* path, CkptHeader& h, std::vector<double>* U, std::vector<double>* phiF) {
    FILE* fp = fopen(path, "rb");
    if (!fp) return fail(HCFD_EIO, std::string("checkpoint: cannot open ") + path);
    auto bad = [&](const char* why) {
        fclose(fp);
        return fail(HCFD_EIO, std::string("checkpoint: ") + why + ": " + path);
    };
    if (fread(&h, sizeof(h), 1, fp) != 1) return bad("short header");
    if (std::memcmp(h.magic, "HCFDCKP1", 8) != 0 || h.version != 1) return bad("not a checkpoint of this library");
    if (h.Nc <= 0 || (h.precision != HCFD_FP64 && h.precision != HCFD_FP32) || (h.has_phiF != 0 && h.has_phiF != 1) ||
        h.steps < 0)
        return bad("corrupt header");
    const size_t n = 4 * (size_t) h.Nc;
    if (U) {
        U->resize(n);
        if (fread(U->data(), 8, n, fp) != n) return bad("short state");
    } else if (fseek(fp, (long) (8 * n), SEEK_CUR) != 0) {
        return bad("short state");
    }
    if (h.has_phiF) {
        if (phiF) {
            phiF->resize(n);
            if (fread(phiF->data(), 8, n, fp) != n) return bad("short limiter values");
        }
    }
    // nothing may follow the declared data
    if (U && (!h.has_phiF || phiF)) {
        char c;
        if (fread(&c, 1, 1, fp) == 1) return bad("trailing bytes");
    }
    fclose(fp);
    return HCFD_OK;
}

}  // namespace hcfd

