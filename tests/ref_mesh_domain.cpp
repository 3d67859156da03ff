// Drop-in check without a GPU: the reference's own Mesh reader (from the reference build)
// feeds GPU::Domain, which must see exactly what GPU::Mesh reads from the same file; then
// GPU::Euler, which creates the device solver, must throw rather than fall back to the CPU.
#include "Mesh.hpp"        // the reference's ::Mesh
#include "hcfd_gpu.hpp"

#include <cstdio>
#include <cstring>

template <class T>
static bool same(const T* a, const T* b, long n) { return n == 0 || std::memcmp(a, b, sizeof(T) * n) == 0; }

int main(int argc, char** argv) {
    if (argc != 2) return 2;
    ::Mesh ref(argv[1]);
    GPU::Mesh ours(argv[1]);
    GPU::Domain a(ref), b(ours);
    const hcfd_mesh_view &x = a.view, &y = b.view;
    bool ok = x.dim == y.dim && x.Nn == y.Nn && x.Nc == y.Nc && x.Nf == y.Nf && x.Ncol == y.Ncol &&
              x.NBCcol == y.NBCcol && a.coltag == b.coltag;
    ok = ok && same(x.coloff, y.coloff, x.Ncol + 1) && same(x.nodes, y.nodes, (long) x.dim * x.Nn) &&
         same(x.fn_con, y.fn_con, 2L * x.Nf) && same(x.fc_con, y.fc_con, 2L * x.Nf) &&
         same(x.cn_off, y.cn_off, x.Nc + 1L) && same(x.cn_con, y.cn_con, (long) x.cn_off[x.Nc]);
    ok = ok && same(ref.cf_off, ours.cf_off, x.Nc + 1L) && same(ref.cf_con, ours.cf_con, (long) ref.cf_off[x.Nc]);
    if (!ok) { std::puts("MISMATCH"); return 1; }
    std::printf("SAME Nc=%d Nf=%d\n", x.Nc, x.Nf);
    try {
        GPU::GaussGreen grads(a);
        GPU::Limiter limiter(a);
        GPU::Flux flux(4, 1.4, a);
        GPU::Euler euler(4, a, flux, grads, limiter);
        std::puts("NO-THROW");
        return 3;
    } catch (const std::runtime_error& e) {
        std::printf("THREW %s\n", e.what());
    }
    return 0;
}
