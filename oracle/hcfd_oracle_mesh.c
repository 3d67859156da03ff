/* TEST INFRASTRUCTURE — input generation for the checker and the CPU baseline, never the product.
 *
 * Writes the triangulated supersonic-wedge mesh as a .hmsh file so that the timed reference
 * arm (bench.py --impl reference) and the CPU baseline read the same mesh as the GPU solver
 * without loading the product library.  It restates the library's generator
 * (hcfd_mesh_generate_wedge and its renumbering in cfd_optimisations_b200/csrc/hcfd_mesh.cpp)
 * step for step, and tests/test_oracle_mesh.py checks the files it writes byte for byte against
 * the library's.  The face conventions follow the reference's pre-processor
 * (interface/Mesh.py:283-378: faces from shared edges, colour = the larger cell tag, ghost cells
 * on the right, faces of a colour sorted by their cell pair) and the file layout the reference
 * reads (src/Mesh.cpp:7-54) and writes (interface/Mesh.py:441-463).
 *
 * Build with FMA contraction off (the library's host code has none), e.g.
 *   gcc -std=gnu11 -O2 -ffp-contract=off -fPIC -shared hcfd_oracle_mesh.c -lm
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { NUM_NATURAL = 0, NUM_RANDOM = 1, NUM_RCM = 2, NUM_MORTON = 3 };

typedef struct {
    int Nn, Nc, Nf, Ncol, NBCcol;
    double* nodes;
    int *cn_off, *cn_con, *ctypes;
    int *fn_con, *fc_con, coloff[6], coltag[5];
    int *cc_off, *cc_con;
} wmesh;

/* SplitMix64, as the library's generator draws it. */
typedef struct { uint64_t s; } splitmix;
static uint64_t sm_next(splitmix* r) {
    uint64_t z = (r->s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static double sm_uniform(splitmix* r) { return (double) (sm_next(r) >> 11) * (1.0 / 9007199254740992.0); }

/* ---- sorting helpers: every key carries a tie-breaker, so qsort gives one order ---- */
typedef struct { uint64_t key; int64_t idx; } kv;
static int kv_cmp(const void* a, const void* b) {
    const kv *x = (const kv*) a, *y = (const kv*) b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return (x->idx > y->idx) - (x->idx < y->idx);
}

/* Neighbour lists from the faces, each sorted ascending. */
static void build_cc(wmesh* m) {
    free(m->cc_off); free(m->cc_con);
    m->cc_off = calloc((size_t) m->Nc + 1, sizeof(int));
    for (int f = 0; f < m->Nf; f++) { m->cc_off[m->fc_con[2 * f] + 1]++; m->cc_off[m->fc_con[2 * f + 1] + 1]++; }
    for (int i = 0; i < m->Nc; i++) m->cc_off[i + 1] += m->cc_off[i];
    m->cc_con = malloc(sizeof(int) * (size_t) m->cc_off[m->Nc]);
    int* cnt = calloc((size_t) m->Nc, sizeof(int));
    for (int f = 0; f < m->Nf; f++) {
        int L = m->fc_con[2 * f], R = m->fc_con[2 * f + 1];
        m->cc_con[m->cc_off[L] + cnt[L]++] = R;
        m->cc_con[m->cc_off[R] + cnt[R]++] = L;
    }
    free(cnt);
    kv* t = malloc(sizeof(kv) * 16);
    for (int i = 0; i < m->Nc; i++) {
        int a = m->cc_off[i], n = m->cc_off[i + 1] - a;
        if (n > 16) { free(t); t = malloc(sizeof(kv) * (size_t) n); }
        for (int k = 0; k < n; k++) { t[k].key = (uint64_t) (uint32_t) m->cc_con[a + k]; t[k].idx = k; }
        qsort(t, (size_t) n, sizeof(kv), kv_cmp);
        for (int k = 0; k < n; k++) m->cc_con[a + k] = (int) t[k].key;
        if (n > 16) { free(t); t = malloc(sizeof(kv) * 16); }
    }
    free(t);
}

/* Faces of each colour sorted by (min cell, max cell); interior faces oriented CL < CR. */
static void sort_faces(wmesh* m) {
    const int F_BC = m->coloff[m->Ncol - m->NBCcol];
    kv* ord = malloc(sizeof(kv) * (size_t) m->Nf);
    for (int f = 0; f < m->Nf; f++) {
        int L = m->fc_con[2 * f], R = m->fc_con[2 * f + 1];
        if (f < F_BC && L > R) { m->fc_con[2 * f] = R; m->fc_con[2 * f + 1] = L; int t = L; L = R; R = t; }
        unsigned lo = (unsigned) (L < R ? L : R), hi = (unsigned) (L < R ? R : L);
        ord[f].key = ((uint64_t) lo << 32) | hi;
        ord[f].idx = f;
    }
    for (int c = 0; c < m->Ncol; c++)
        qsort(ord + m->coloff[c], (size_t) (m->coloff[c + 1] - m->coloff[c]), sizeof(kv), kv_cmp);
    int* fc = malloc(sizeof(int) * 2 * (size_t) m->Nf);
    int* fn = malloc(sizeof(int) * 2 * (size_t) m->Nf);
    for (int k = 0; k < m->Nf; k++) {
        int f = (int) ord[k].idx;
        fc[2 * k] = m->fc_con[2 * f]; fc[2 * k + 1] = m->fc_con[2 * f + 1];
        fn[2 * k] = m->fn_con[2 * f]; fn[2 * k + 1] = m->fn_con[2 * f + 1];
    }
    free(m->fc_con); free(m->fn_con); free(ord);
    m->fc_con = fc; m->fn_con = fn;
}

/* perm[new] = old. */
static void apply_cell_perm(wmesh* m, const int* perm) {
    int* inv = malloc(sizeof(int) * (size_t) m->Nc);
    for (int i = 0; i < m->Nc; i++) inv[perm[i]] = i;
    int* off = malloc(sizeof(int) * ((size_t) m->Nc + 1));
    int* con = malloc(sizeof(int) * (size_t) m->cn_off[m->Nc]);
    int* ct = malloc(sizeof(int) * (size_t) m->Nc);
    off[0] = 0;
    for (int i = 0; i < m->Nc; i++) {
        int o = perm[i], n = m->cn_off[o + 1] - m->cn_off[o];
        memcpy(con + off[i], m->cn_con + m->cn_off[o], sizeof(int) * (size_t) n);
        off[i + 1] = off[i] + n;
        ct[i] = m->ctypes[o];
    }
    free(m->cn_off); free(m->cn_con); free(m->ctypes);
    m->cn_off = off; m->cn_con = con; m->ctypes = ct;
    for (int k = 0; k < 2 * m->Nf; k++) m->fc_con[k] = inv[m->fc_con[k]];
    free(inv);
    sort_faces(m);
    build_cc(m);
}

static int* random_perm(int n, uint64_t seed) {
    int* p = malloc(sizeof(int) * (size_t) n);
    for (int i = 0; i < n; i++) p[i] = i;
    splitmix r = {seed ^ 0xA5A5A5A5DEADBEEFULL};
    for (int i = n - 1; i > 0; i--) {
        int j = (int) (sm_next(&r) % (uint64_t) (i + 1));
        int t = p[i]; p[i] = p[j]; p[j] = t;
    }
    return p;
}

/* BFS from s over cells not yet numbered; returns a minimum-degree cell of the last level
 * (the first one met in BFS order among equals). */
static int bfs_last(const wmesh* m, const int* deg, const char* seen, int* level, int* q, int s) {
    int head = 0, tail = 0, maxl = 0;
    q[tail++] = s; level[s] = 0;
    while (head < tail) {
        int c = q[head++];
        for (int k = m->cc_off[c]; k < m->cc_off[c + 1]; k++) {
            int d = m->cc_con[k];
            if (seen[d] || level[d] >= 0) continue;
            level[d] = level[c] + 1;
            if (level[d] > maxl) maxl = level[d];
            q[tail++] = d;
        }
    }
    int best = -1;
    for (int i = 0; i < tail; i++) { int c = q[i]; if (level[c] == maxl && (best < 0 || deg[c] < deg[best])) best = c; }
    for (int i = 0; i < tail; i++) level[q[i]] = -1;
    return best;
}

/* Reverse Cuthill-McKee over the face adjacency: per connected component, a BFS from a
 * pseudo-peripheral cell (up to three BFS sweeps from the minimum-degree cell), neighbours
 * in increasing (degree, index), the final order reversed. */
static int* rcm_perm(const wmesh* m) {
    const int n = m->Nc;
    int* deg = malloc(sizeof(int) * (size_t) n);
    for (int i = 0; i < n; i++) deg[i] = m->cc_off[i + 1] - m->cc_off[i];
    kv* bydeg = malloc(sizeof(kv) * (size_t) n);
    for (int i = 0; i < n; i++) { bydeg[i].key = (uint64_t) deg[i]; bydeg[i].idx = i; }
    qsort(bydeg, (size_t) n, sizeof(kv), kv_cmp);
    char* seen = calloc((size_t) n, 1);
    int* level = malloc(sizeof(int) * (size_t) n);
    for (int i = 0; i < n; i++) level[i] = -1;
    int* q = malloc(sizeof(int) * (size_t) n);
    int* order = malloc(sizeof(int) * (size_t) n);
    int no = 0;
    kv nb[64];
    for (int i0 = 0; i0 < n; i0++) {
        int start0 = (int) bydeg[i0].idx;
        if (seen[start0]) continue;
        int s = start0;
        for (int it = 0; it < 3; it++) { int t = bfs_last(m, deg, seen, level, q, s); if (t == s) break; s = t; }
        int head = no, tail = no;
        order[tail++] = s; seen[s] = 1;
        while (head < tail) {
            int c = order[head++];
            int nn = 0;
            for (int k = m->cc_off[c]; k < m->cc_off[c + 1]; k++) {
                int d = m->cc_con[k];
                if (!seen[d]) { nb[nn].key = (uint64_t) deg[d]; nb[nn].idx = d; nn++; }
            }
            qsort(nb, (size_t) nn, sizeof(kv), kv_cmp);
            for (int k = 0; k < nn; k++) { seen[nb[k].idx] = 1; order[tail++] = (int) nb[k].idx; }
        }
        no = tail;
    }
    for (int i = 0; i < n / 2; i++) { int t = order[i]; order[i] = order[n - 1 - i]; order[n - 1 - i] = t; }
    free(deg); free(bydeg); free(seen); free(level); free(q);
    return order;
}

static uint64_t spread32(uint64_t x) {
    x &= 0xFFFFFFFFULL;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFULL;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFULL;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0FULL;
    x = (x | (x << 2)) & 0x3333333333333333ULL;
    x = (x | (x << 1)) & 0x5555555555555555ULL;
    return x;
}

/* Cells by the Morton key of their vertex-average centre, quantised to 2^31 steps over the
 * node bounding box; equal keys keep their order. */
static int* morton_perm(const wmesh* m) {
    double lo[2] = {1e300, 1e300}, hi[2] = {-1e300, -1e300};
    for (int i = 0; i < m->Nn; i++)
        for (int d = 0; d < 2; d++) {
            double v = m->nodes[2 * i + d];
            if (v < lo[d]) lo[d] = v;
            if (v > hi[d]) hi[d] = v;
        }
    kv* k = malloc(sizeof(kv) * (size_t) m->Nc);
    for (int c = 0; c < m->Nc; c++) {
        double x[2] = {0, 0};
        int nn = m->cn_off[c + 1] - m->cn_off[c];
        for (int j = m->cn_off[c]; j < m->cn_off[c + 1]; j++)
            for (int d = 0; d < 2; d++) x[d] += m->nodes[2 * m->cn_con[j] + d] / nn;
        uint64_t qd[2];
        for (int d = 0; d < 2; d++) {
            double t = (hi[d] > lo[d]) ? (x[d] - lo[d]) / (hi[d] - lo[d]) : 0.0;
            t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
            qd[d] = (uint64_t) (t * 2147483647.0);
        }
        k[c].key = spread32(qd[0]) | (spread32(qd[1]) << 1);
        k[c].idx = c;
    }
    qsort(k, (size_t) m->Nc, sizeof(kv), kv_cmp);
    int* p = malloc(sizeof(int) * (size_t) m->Nc);
    for (int c = 0; c < m->Nc; c++) p[c] = (int) k[c].idx;
    free(k);
    return p;
}

/* Faces from shared edges (each edge in exactly two cells); colour = the larger tag of the
 * two cells; ghost cells (tag > 0) on the right; interior faces with the lower index on the
 * left.  Faces are grouped by colour in the order of their edge keys, then sorted. */
static int build_faces(wmesh* m, const int* ctag) {
    size_t ne = (size_t) m->cn_off[m->Nc];
    kv* e = malloc(sizeof(kv) * ne);
    size_t k = 0;
    for (int c = 0; c < m->Nc; c++) {
        int a = m->cn_off[c], n = m->cn_off[c + 1] - a;
        int edges = n == 2 ? 1 : n;
        for (int j = 0; j < edges; j++) {
            int u = m->cn_con[a + j], v = m->cn_con[a + (j + 1) % n];
            e[k].key = ((uint64_t) (unsigned) (u < v ? u : v) << 32) | (unsigned) (u < v ? v : u);
            e[k].idx = c;
            k++;
        }
    }
    ne = k;
    qsort(e, ne, sizeof(kv), kv_cmp);
    int* fcol = malloc(sizeof(int) * ne);
    int* fc = malloc(sizeof(int) * ne * 2);
    int* fn = malloc(sizeof(int) * ne * 2);
    int nf = 0, bad = 0;
    for (size_t i = 0; i < ne;) {
        size_t j = i;
        while (j < ne && e[j].key == e[i].key) j++;
        if (j - i != 2) { bad = 1; break; }
        int c1 = (int) e[i].idx, c2 = (int) e[i + 1].idx;
        int col = ctag[c1] > ctag[c2] ? ctag[c1] : ctag[c2];
        if (ctag[c1] > 0 && ctag[c2] > 0) { bad = 1; break; }
        int L = c1, R = c2;
        if (ctag[L] > ctag[R] || (col == 0 && L > R)) { int t = L; L = R; R = t; }
        fcol[nf] = col;
        fc[2 * nf] = L; fc[2 * nf + 1] = R;
        fn[2 * nf] = (int) (e[i].key >> 32); fn[2 * nf + 1] = (int) (e[i].key & 0xFFFFFFFFULL);
        nf++;
        i = j;
    }
    free(e);
    if (bad) { free(fcol); free(fc); free(fn); return -1; }
    m->Nf = nf;
    m->Ncol = 5;
    m->fc_con = malloc(sizeof(int) * 2 * (size_t) nf);
    m->fn_con = malloc(sizeof(int) * 2 * (size_t) nf);
    int f = 0;
    m->coloff[0] = 0;
    for (int c = 0; c < 5; c++) {
        m->coltag[c] = c;
        for (int i = 0; i < nf; i++) {
            if (fcol[i] != c) continue;
            m->fc_con[2 * f] = fc[2 * i]; m->fc_con[2 * f + 1] = fc[2 * i + 1];
            m->fn_con[2 * f] = fn[2 * i]; m->fn_con[2 * f + 1] = fn[2 * i + 1];
            f++;
        }
        m->coloff[c + 1] = f;
    }
    free(fcol); free(fc); free(fn);
    sort_faces(m);
    build_cc(m);
    return 0;
}

static void free_mesh(wmesh* m) {
    free(m->nodes); free(m->cn_off); free(m->cn_con); free(m->ctypes);
    free(m->fn_con); free(m->fc_con); free(m->cc_off); free(m->cc_con);
}

static int write_hmsh(const wmesh* m, const char* path) {
    static const char names[] = "upper\0lower\0inlet\0outlet";
    const int nch = (int) sizeof(names);   /* 25: four NUL-terminated names */
    FILE* fp = fopen(path, "wb");
    if (!fp) return -2;
    int N[8] = {2, m->Nn, m->Ncol, m->NBCcol, m->Nc, m->Nf, 4, nch};
    int ok = fwrite(N, 4, 8, fp) == 8;
    ok = ok && fwrite(names, 1, (size_t) nch, fp) == (size_t) nch;
    ok = ok && fwrite(m->coltag, 4, 5, fp) == 5;
    ok = ok && fwrite(m->coloff, 4, 6, fp) == 6;
    ok = ok && fwrite(m->nodes, 8, 2 * (size_t) m->Nn, fp) == 2 * (size_t) m->Nn;
    ok = ok && fwrite(m->fn_con, 4, 2 * (size_t) m->Nf, fp) == 2 * (size_t) m->Nf;
    ok = ok && fwrite(m->fc_con, 4, 2 * (size_t) m->Nf, fp) == 2 * (size_t) m->Nf;
    ok = ok && fwrite(m->cn_off, 4, (size_t) m->Nc + 1, fp) == (size_t) m->Nc + 1;
    ok = ok && fwrite(m->cn_con, 4, (size_t) m->cn_off[m->Nc], fp) == (size_t) m->cn_off[m->Nc];
    ok = ok && fwrite(m->cc_off, 4, (size_t) m->Nc + 1, fp) == (size_t) m->Nc + 1;
    ok = ok && fwrite(m->cc_con, 4, (size_t) m->cc_off[m->Nc], fp) == (size_t) m->cc_off[m->Nc];
    ok = ok && fwrite(m->ctypes, 4, (size_t) m->Nc, fp) == (size_t) m->Nc;
    ok = (fclose(fp) == 0) && ok;
    return ok ? 0 : -2;
}

/* The wedge: x in [0, length], top wall y = height, bottom y_b(x) = max(0, (x - x_ramp) tan
 * theta); nodes mapped vertically between y_b and the top, interior nodes jittered by
 * U(+-jitter) of the local spacing; each quad split into two triangles by a seeded coin flip;
 * boundary line cells (ghosts) tagged 1 upper, 2 lower, 3 inlet, 4 outlet.  Returns 0, -1 for
 * bad arguments or an inverted triangle, -2 for an I/O error. */
int hcfd_oracle_wedge_hmsh(int nx, int ny, double length, double height, double x_ramp, double theta_deg,
                           double jitter, unsigned long long seed, int numbering, const char* path) {
    if (nx < 3 || ny < 3 || (long long) nx * ny > (1LL << 29) || !(length > 0) || !(height > 0) ||
        !(jitter >= 0 && jitter < 0.5) || !(theta_deg >= 0 && theta_deg < 60) || numbering < 0 || numbering > 3 ||
        !path)
        return -1;
    wmesh m;
    memset(&m, 0, sizeof(m));
    m.Nn = nx * ny;
    m.NBCcol = 4;
    m.nodes = malloc(sizeof(double) * 2 * (size_t) m.Nn);
    const double tanth = tan(theta_deg * M_PI / 180.0);
    const double hx = length / (nx - 1);
    splitmix rng = {seed};
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            double x = length * i / (nx - 1);
            const double ramp = (x - x_ramp) * tanth;
            double yb = 0.0 < ramp ? ramp : 0.0;
            if (yb >= height) { free_mesh(&m); return -1; }
            double y = yb + (height - yb) * j / (ny - 1);
            if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && jitter > 0) {
                double hy = (height - yb) / (ny - 1);
                x += (2.0 * sm_uniform(&rng) - 1.0) * jitter * hx;
                y += (2.0 * sm_uniform(&rng) - 1.0) * jitter * hy;
            }
            m.nodes[2 * (j * nx + i)] = x;
            m.nodes[2 * (j * nx + i) + 1] = y;
        }
    const int ntri = 2 * (nx - 1) * (ny - 1), ng = 2 * (nx - 1) + 2 * (ny - 1);
    m.Nc = ntri + ng;
    m.cn_off = malloc(sizeof(int) * ((size_t) m.Nc + 1));
    m.cn_con = malloc(sizeof(int) * (3 * (size_t) ntri + 2 * (size_t) ng));
    m.ctypes = malloc(sizeof(int) * (size_t) m.Nc);
    int* ctag = malloc(sizeof(int) * (size_t) m.Nc);
    int c = 0, k = 0;
    m.cn_off[0] = 0;
#define PUSH3(a, b, d, tag) do { m.cn_con[k++] = (a); m.cn_con[k++] = (b); m.cn_con[k++] = (d); \
        ctag[c] = (tag); m.ctypes[c] = 2; m.cn_off[++c] = k; } while (0)
#define PUSH2(a, b, tag) do { m.cn_con[k++] = (a); m.cn_con[k++] = (b); \
        ctag[c] = (tag); m.ctypes[c] = 1; m.cn_off[++c] = k; } while (0)
#define NODE(i, j) ((j) * nx + (i))
    for (int j = 0; j < ny - 1; j++)
        for (int i = 0; i < nx - 1; i++) {
            int a = NODE(i, j), b = NODE(i + 1, j), cc = NODE(i + 1, j + 1), d = NODE(i, j + 1);
            if (sm_next(&rng) >> 63) { PUSH3(a, b, cc, 0); PUSH3(a, cc, d, 0); }
            else                     { PUSH3(a, b, d, 0);  PUSH3(b, cc, d, 0); }
        }
    for (int i = 0; i < nx - 1; i++) PUSH2(NODE(i, ny - 1), NODE(i + 1, ny - 1), 1);
    for (int i = 0; i < nx - 1; i++) PUSH2(NODE(i, 0), NODE(i + 1, 0), 2);
    for (int j = 0; j < ny - 1; j++) PUSH2(NODE(0, j), NODE(0, j + 1), 3);
    for (int j = 0; j < ny - 1; j++) PUSH2(NODE(nx - 1, j), NODE(nx - 1, j + 1), 4);
#undef PUSH3
#undef PUSH2
#undef NODE
    for (int t = 0; t < ntri; t++) {
        const int* n3 = m.cn_con + m.cn_off[t];
        double ax = m.nodes[2 * n3[0]], ay = m.nodes[2 * n3[0] + 1];
        double bx = m.nodes[2 * n3[1]], by = m.nodes[2 * n3[1] + 1];
        double cx = m.nodes[2 * n3[2]], cy = m.nodes[2 * n3[2] + 1];
        if ((bx - ax) * (cy - ay) - (by - ay) * (cx - ax) <= 0) { free(ctag); free_mesh(&m); return -1; }
    }
    int rc = build_faces(&m, ctag);
    free(ctag);
    if (rc == 0 && numbering != NUM_NATURAL) {
        int* p = numbering == NUM_RANDOM ? random_perm(m.Nc, seed) : numbering == NUM_RCM ? rcm_perm(&m) : morton_perm(&m);
        apply_cell_perm(&m, p);
        free(p);
    }
    if (rc == 0) rc = write_hmsh(&m, path);
    free_mesh(&m);
    return rc;
}
